// Host-side harness for the device minimiser controller: runs the same
// minimize_control_core that k_minimize_control runs on the GPU, with the
// per-cell update of the RHS_MINIMIZE epilogue done here in FP64 on the
// oracle's effective field.  With identical arithmetic underneath, its report
// and final state must equal the oracle's restatement of minimize_damping_only.
// Test infrastructure only.
#include <cmath>
#include <cstring>
#include <vector>

#include "../../oracle/oracle.h"
#include "../../llg-sim_b200/csrc/minimize_dev.cuh"

using namespace llg;

extern "C" int harness_minimize(const orc_grid* g, const orc_material* mat, const uint8_t* mask, double* m,
                                const orc_params* p, int fmask, const orc_minimize_settings* st,
                                orc_minimize_report* rep) {
    const int64_t n = g->nx * g->ny;
    orc_solver* s = orc_solver_create(g, mat, mask);
    MinimizeSettingsDev S{};
    S.thr = st->torque_threshold;
    S.lambda0 = st->lambda0;
    S.lambda_min = st->lambda_min;
    S.lambda_max = st->lambda_max;
    S.grow = st->grow;
    S.shrink = st->shrink;
    S.stall_rel = st->stall_rel;
    S.dm_stop = st->dm_stop;
    S.gate = st->dm_torque_gate;
    S.gate_max = st->dm_torque_gate_max;
    S.max_iters = st->max_iters;
    S.stall_iters = st->stall_iters;
    S.min_iters_before_stall = st->min_iters_before_stall;
    S.dm_samples = st->dm_samples;
    S.dm_min_iters = st->dm_min_iters;
    S.has_dm_stop = st->has_dm_stop;
    S.has_gate = st->has_dm_torque_gate;
    S.has_gate_max = st->has_dm_torque_gate_max;
    MinimizeStateDev M;
    minimize_state_init(M, S, (double)n);
    std::vector<double> b(3 * n);
    long long guard = 0;
    while (!M.done) {
        if (++guard > S.max_iters + 8) {
            orc_solver_destroy(s);
            return 1;
        }
        orc_build_h_eff(s, m, p->b_ext, fmask, b.data());
        double tmax = 0.0, tsum = 0.0, dmx = 0.0;
        const double lam = M.lambda;
        for (int64_t i = 0; i < n; ++i) {
            const double m0 = m[3 * i], m1 = m[3 * i + 1], m2 = m[3 * i + 2];
            const double b0 = b[3 * i], b1 = b[3 * i + 1], b2 = b[3 * i + 2];
            const double q0 = m1 * b2 - m2 * b1, q1 = m2 * b0 - m0 * b2, q2 = m0 * b1 - m1 * b0;
            const double tm = std::sqrt(q0 * q0 + q1 * q1 + q2 * q2);
            tsum += tm;
            tmax = std::fmax(tmax, tm);
            double x = m0 + lam * (q1 * m2 - q2 * m1);
            double y = m1 + lam * (q2 * m0 - q0 * m2);
            double z = m2 + lam * (q0 * m1 - q1 * m0);
            const double n2 = x * x + y * y + z * z;
            if (n2 > 0.0) {
                const double inv = 1.0 / std::sqrt(n2);
                x *= inv;
                y *= inv;
                z *= inv;
            }
            const double ex = x - m0, ey = y - m1, ez = z - m2;
            dmx = std::fmax(dmx, std::sqrt(ex * ex + ey * ey + ez * ez));
            m[3 * i] = x;
            m[3 * i + 1] = y;
            m[3 * i + 2] = z;
        }
        minimize_control_core(M, S, tmax, tsum, dmx);
    }
    rep->iters = M.iters;
    rep->converged = M.converged;
    rep->stalled = M.stalled;
    rep->dm_converged = M.dm_converged;
    rep->reserved = 0;
    rep->final_torque = M.final_torque;
    rep->final_max_dm = M.final_max_dm;
    rep->final_tmean = M.final_tmean;
    rep->final_lambda = M.final_lambda;
    orc_solver_destroy(s);
    return 0;
}
