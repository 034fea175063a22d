// Host-side harness for the device relax controller: runs the same
// relax_control_core state machine that the GPU runs, but executes its
// requests (energy, torque rebuild, RK23 relax attempt) with the FP64 oracle.
// With identical arithmetic underneath, its report and final state must equal
// the oracle's own relax_with_report restatement.  Test infrastructure only.
#include <cmath>
#include <cstring>
#include <vector>

#include "../../oracle/oracle.h"
#include "../../llg-sim_b200/csrc/relax_dev.cuh"

using namespace llg;

namespace {
struct HostStep {
    int req = REQ_NONE, accepted = 0, err_code = 0, active = 1;
    double red[RED_NSLOT] = {};
    double max_err = 0, headroom = 0, dt_min = 0, dt_max = 0;
    long long attempts_left = -1, target_acc = -1;
};

void torque_stats(int64_t n, const double* m, const double* b, double* red) {
    double tmax = 0, tsum = 0, tsum2 = 0;
    for (int64_t i = 0; i < n; ++i) {
        const double* a = &m[3 * i];
        const double* c = &b[3 * i];
        double t0 = a[1] * c[2] - a[2] * c[1], t1 = a[2] * c[0] - a[0] * c[2], t2 = a[0] * c[1] - a[1] * c[0];
        double s2 = t0 * t0 + t1 * t1 + t2 * t2, s = std::sqrt(s2);
        if (s > tmax) tmax = s;
        tsum += s;
        tsum2 += s2;
    }
    red[RED_TMAX] = tmax;
    red[RED_TSUM] = tsum;
    red[RED_TSUM2] = tsum2;
}
}  // namespace

extern "C" int harness_relax(const orc_grid* g, const orc_material* mat, const uint8_t* mask, double* m,
                             orc_params* p, int fmask, const orc_relax_settings* st, orc_relax_report* rep,
                             long long max_iters) {
    const int64_t n = g->nx * g->ny;
    orc_solver* s = orc_solver_create(g, mat, mask);
    RelaxSettingsDev S{};
    S.max_err = st->max_err;
    S.headroom = st->headroom;
    S.dt_min = st->dt_min;
    S.dt_max = st->dt_max;
    S.rel_energy_tol = st->rel_energy_tol;
    S.thr = st->torque_threshold;
    S.plateau_rel = st->torque_plateau_rel;
    S.plateau_abs = st->torque_plateau_abs;
    S.tighten_factor = st->tighten_factor;
    S.tighten_floor = st->tighten_floor;
    S.gate = st->final_torque_gate;
    S.gate_max = st->final_torque_gate_max;
    S.energy_stride = st->energy_stride;
    S.check_stride = st->torque_check_stride;
    S.plateau_checks = st->torque_plateau_checks;
    S.plateau_min_checks = st->torque_plateau_min_checks;
    S.max_acc = st->max_accepted_steps;
    S.gate_extra = st->gate_max_extra_accepted_steps;
    S.gate_plateau_fails = st->gate_plateau_fails;
    S.phase1 = st->phase1_enabled;
    S.phase2 = st->phase2_enabled;
    S.metric = st->torque_metric;
    S.has_thr = st->has_torque_threshold;
    S.has_gate = st->has_final_torque_gate;
    S.has_gmax = st->has_final_torque_gate_max;
    RelaxStateDev R;
    std::memset(&R, 0, sizeof(R));
    R.pc = RP_START;
    R.last_stage = -1;
    R.max_err = st->max_err;
    R.n_cells = (double)n;
    p->dt = std::fmin(std::fmax(p->dt, st->dt_min), st->dt_max);
    orc_solver_invalidate(s);
    HostStep hs;
    std::vector<double> b(3 * n);
    relax_control_core(&hs, R, S);
    long long it = 0;
    for (; !R.done && it < max_iters; ++it) {
        if (hs.req == REQ_ENERGY) {
            orc_energy e;
            orc_energy_breakdown(s, m, p->b_ext, &e);
            hs.red[RED_E_EX] = e.exchange;
            hs.red[RED_E_AN] = e.anisotropy;
            hs.red[RED_E_ZEE] = e.zeeman;
            hs.red[RED_E_DMI] = e.dmi;
            hs.red[RED_E_DEMAG] = e.demag;
        } else if (hs.req == REQ_TORQUE) {
            orc_build_h_eff(s, m, p->b_ext, fmask, b.data());
            torque_stats(n, m, b.data(), hs.red);
        } else if (hs.req == REQ_STEP) {
            double eps, dtu;
            int acc;
            orc_step_rk23_relax(s, m, p, fmask, hs.max_err, hs.headroom, hs.dt_min, hs.dt_max, &eps, &acc, &dtu);
            hs.accepted = acc;
            if (acc) {
                orc_build_h_eff(s, m, p->b_ext, fmask, b.data());
                torque_stats(n, m, b.data(), hs.red);
            }
        }
        relax_control_core(&hs, R, S);
    }
    orc_solver_destroy(s);
    rep->accepted_steps = R.accepted;
    rep->rejected_steps = R.rejected;
    rep->torque_checks = R.checks;
    rep->torque_field_rebuilds = R.rebuilds;
    rep->stop_reason = R.stop_reason;
    rep->last_stage_stop = R.last_stage;
    rep->has_final_torque = R.has_ft;
    rep->final_torque = R.ft;
    rep->has_final_torque_max = R.has_ftm;
    rep->final_torque_max = R.ftm;
    rep->final_max_err = R.max_err;
    rep->final_dt = p->dt;
    return R.done ? 0 : -3;
}
