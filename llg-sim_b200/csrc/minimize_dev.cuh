// minimize_dev.cuh — minimize_damping_only (minimize.rs:107-369) as a per-film
// device controller.
//
// One minimiser iteration of the replayed graph is a field evaluation with
// RhsMode RHS_MINIMIZE (the effective field, the damping-only update of every
// cell written to the other parity buffer, the FP64 block reductions of
// max |m x B| and sum |m x B|, and max |m' - m| through the film's error-norm
// accumulator), the deterministic per-film finalisation of the
// reductions, and k_minimize_control, which adopts the update and runs the
// iteration's decisions: torque threshold, the dM stop with its torque gates,
// the lambda controller and the stall counter.  A finished film drops its
// REQ_MINIMIZE request, so the rest of the graph skips it.
#pragma once
#include <cmath>

#include "types.cuh"

#ifdef __CUDACC__
#define LLG_HD __host__ __device__
#else
#define LLG_HD
#endif

namespace llg {

// MinimizeSettings (minimize.rs:20-63); the Option fields as has_* flags.
struct MinimizeSettingsDev {
    double thr, lambda0, lambda_min, lambda_max, grow, shrink, stall_rel, dm_stop, gate, gate_max;
    long long max_iters, stall_iters, min_iters_before_stall, dm_samples, dm_min_iters;
    int has_dm_stop, has_gate, has_gate_max;
};

struct MinimizeStateDev {
    double lambda, t_prev_mean, last_max_dm, last_tmax, last_tmean;
    long long it, stall_count;
    // Trailing run of dM samples below dm_stop.  The reference keeps the last
    // dm_samples values in a queue and stops when the queue is full and every
    // value is below dm_stop, which holds exactly when the last dm_samples
    // pushed values are all below it.
    long long dm_run;
    double n_cells;
    int done;
    // MinimizeReport (minimize.rs:94-104)
    int converged, stalled, dm_converged;
    long long iters;
    double final_torque, final_max_dm, final_tmean, final_lambda;
};

LLG_HD inline void minimize_state_init(MinimizeStateDev& M, const MinimizeSettingsDev& S, double n_cells) {
    M.lambda = S.lambda0;
    M.t_prev_mean = INFINITY;
    M.last_max_dm = INFINITY;
    M.last_tmax = INFINITY;
    M.last_tmean = INFINITY;
    M.it = 0;
    M.stall_count = 0;
    M.dm_run = 0;
    M.n_cells = n_cells;
    M.done = 0;
    M.converged = M.stalled = M.dm_converged = 0;
    M.iters = 0;
    M.final_torque = M.final_max_dm = M.final_tmean = 0.0;
    M.final_lambda = S.lambda0;
    if (S.max_iters <= 0) {
        // the loop body never runs (minimize.rs:359-368)
        M.done = 1;
        M.iters = 0;
        M.final_torque = INFINITY;
        M.final_max_dm = INFINITY;
        M.final_tmean = INFINITY;
    }
}

LLG_HD inline void minimize_finish(MinimizeStateDev& M, long long iters, double ft, int conv, int stalled, double mdm,
                                   int dmc, double tmean) {
    M.done = 1;
    M.iters = iters;
    M.final_torque = ft;
    M.converged = conv;
    M.stalled = stalled;
    M.final_max_dm = mdm;
    M.dm_converged = dmc;
    M.final_tmean = tmean;
    M.final_lambda = M.lambda;
}

// Consumes the statistics of the update just applied (minimize.rs:258-356).
// Returns 1 when the minimiser has finished.
LLG_HD inline int minimize_control_core(MinimizeStateDev& M, const MinimizeSettingsDev& S, double tmax, double tsum,
                                        double max_dm) {
    using std::fabs;
    using std::fmax;
    using std::fmin;
    const long long it = M.it;
    const double tmean = tsum / fmax(M.n_cells, 1.0);
    M.last_tmean = tmean;
    if (tmax < S.thr) {
        minimize_finish(M, it + 1, tmax, 1, 0, max_dm, 0, tmean);
        return 1;
    }
    M.last_max_dm = max_dm;
    M.last_tmax = tmax;
    if (S.has_dm_stop && it + 1 >= S.dm_min_iters) {
        M.dm_run = max_dm < S.dm_stop ? M.dm_run + 1 : 0;
        const long long need = S.dm_samples > 1 ? S.dm_samples : 1;
        if (M.dm_run >= need) {
            const bool mean_ok = !S.has_gate || tmean <= S.gate;
            const bool max_ok = !S.has_gate_max || tmax <= S.gate_max;
            minimize_finish(M, it + 1, tmax, (mean_ok && max_ok) ? 1 : 0, 0, max_dm, 1, tmean);
            return 1;
        }
    }
    // lambda from the change of the mean torque (minimize.rs:321-326)
    if (tmean < M.t_prev_mean) M.lambda = fmin(M.lambda * S.grow, S.lambda_max);
    else M.lambda = fmax(M.lambda * S.shrink, S.lambda_min);
    // stall counter (minimize.rs:328-337)
    if (it + 1 >= S.min_iters_before_stall && std::isfinite(M.t_prev_mean)) {
        const double good = M.t_prev_mean - tmean;
        const double need = S.stall_rel * fmax(fabs(M.t_prev_mean), 1e-30);
        if (good <= need) M.stall_count += 1;
        else M.stall_count = 0;
    }
    if (M.stall_count >= S.stall_iters) {
        minimize_finish(M, it + 1, tmax, 0, 1, M.last_max_dm, 0, tmean);
        return 1;
    }
    M.t_prev_mean = tmean;
    M.it = it + 1;
    if (M.it >= S.max_iters) {
        minimize_finish(M, S.max_iters, M.last_tmax, 0, 0, M.last_max_dm, 0, M.last_tmean);
        return 1;
    }
    return 0;
}

#ifdef __CUDACC__
// Arms the films of a minimiser call: REQ_MINIMIZE and the first lambda.
__global__ void k_minimize_begin(FilmDev* films, const MinimizeStateDev* ms_all, int nfilms) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfilms) return;
    StepState* st = films[f].st;
    const MinimizeStateDev& M = ms_all[f];
    st->active = M.done ? 0 : 1;
    st->req = M.done ? REQ_NONE : REQ_MINIMIZE;
    st->lam = M.lambda;
}

// One thread per film, after the RHS_MINIMIZE evaluation and k_finalize.
__global__ void k_minimize_control(FilmDev* films, MinimizeStateDev* ms_all, int nfilms, MinimizeSettingsDev S) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfilms) return;
    StepState* st = films[f].st;
    if (!st->active || st->req != REQ_MINIMIZE) return;
    MinimizeStateDev& M = ms_all[f];
    st->cur ^= 1;  // the updated state is the film's state from here on
    // max |m' - m| arrives in the error-norm accumulator (max of non-negative bit patterns)
    const double dmx = __longlong_as_double((long long)st->err_bits);
    st->err_bits = 0ull;
    const double tmax = st->red[RED_TMAX], tsum = st->red[RED_TSUM];
    if (minimize_control_core(M, S, tmax, tsum, dmx)) {
        st->req = REQ_NONE;
        st->active = 0;
    }
    st->lam = M.lambda;
}
#endif

}  // namespace llg
