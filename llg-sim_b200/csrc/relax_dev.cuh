// relax_dev.cuh — relax_with_report (relax.rs:334-768) as a per-film device
// state machine.
//
// Each relax iteration of the replayed graph executes at most one request per
// film — an energy evaluation (compute_total_energy, energy.rs:287), a torque
// rebuild (torque_metric_rebuild, relax.rs:192) or one RK23 relax attempt
// (llg.rs:278) — gated by StepState::req, and then runs k_relax_control, which
// consumes the result and advances the film's program counter to the next
// request.  Films advance independently; a finished film goes inactive.
#pragma once
#include <cmath>

#include "types.cuh"

#ifdef __CUDACC__
#define LLG_HD __host__ __device__
#else
#define LLG_HD
#endif

namespace llg {

// Relax settings (RelaxSettings, relax.rs:73-105), shared by all films.
struct RelaxSettingsDev {
    double max_err, headroom, dt_min, dt_max, rel_energy_tol, thr, plateau_rel, plateau_abs, tighten_factor,
        tighten_floor, gate, gate_max;
    long long energy_stride, check_stride, plateau_checks, plateau_min_checks, max_acc, gate_extra, gate_plateau_fails;
    int phase1, phase2, metric, has_thr, has_gate, has_gmax;
};

// Program counters.
enum RelaxPc : int {
    RP_START = 0, RP_P1_E0, RP_P1_ADV, RP_P1_E1, RP_P2_START, RP_STAGE_T0, RP_STAGE_LOOP, RP_STAGE_ADV,
    RP_STAGE_TNEW, RP_STAGE_END, RP_FINAL_T, RP_GATE_LOOP, RP_GATE_TMETRIC, RP_GATE_TMAX, RP_GATE_ADV,
    RP_FAIL_P1, RP_FAIL_STAGE, RP_FAIL_GATE, RP_DONE
};

struct RelaxStateDev {
    int pc;
    int ret_pc;            // where an advance()/torque_now() returns to
    int adv_active;        // inside advance()
    int adv_fail_pc;       // how a failed advance finishes
    long long adv_target;
    int t_metric;          // metric requested from torque_now
    int last_b_eff_valid;  // torque stats of the resident state are current (relax.rs:206-227)
    double max_err;
    long long accepted, rejected, checks, rebuilds;
    double e0, value;
    double t_prev, t_metric_v, t_max_v;
    float t_prev_f32;
    int f32mode;
    long long fails, comparisons;
    long long gate_start, gfails;
    double gate_last_t;
    double tcache_max, tcache_sum, tcache_sum2;
    int last_stage, has_ft, has_ftm, stop_reason, done;
    double ft, ftm;
    double n_cells;
};

LLG_HD inline double torque_from(int metric, double tmax, double tsum, double tsum2, double n) {
    switch (metric) {
        case 0: return tmax;
        case 1: return tsum / fmax(n, 1.0);
        case 2: return sqrt(tsum2 / fmax(n, 1.0));
        default: return tsum2 / fmax(n, 1.0);
    }
}

// One control step of one film: consume the result of the request executed in
// this iteration (st->req), then run the program until it issues the next
// request or finishes.  ST provides the StepState fields used here; the same
// code runs on the device and in the host-side test harness.
template <typename ST>
LLG_HD void relax_control_core(ST* st, RelaxStateDev& R, const RelaxSettingsDev& S) {
    using std::fabs;
    using std::fmax;
    using std::sqrt;
    if (R.done || !st->active) return;
    const int req_done = st->req;  // the request executed in this iteration (if any)
    st->req = REQ_NONE;

    // --- consume the result of the executed request ---
    if (req_done == REQ_STEP) {
        if (st->err_code) {  // non-finite: retire the film
            R.stop_reason = 0;
            R.done = 1;
            st->active = 0;
            return;
        }
        if (st->accepted) {
            R.accepted += 1;
            R.last_b_eff_valid = 1;
            R.tcache_max = st->red[RED_TMAX];
            R.tcache_sum = st->red[RED_TSUM];
            R.tcache_sum2 = st->red[RED_TSUM2];
        } else {
            R.rejected += 1;
            R.last_b_eff_valid = 0;
        }
    } else if (req_done == REQ_ENERGY) {
        R.value = st->red[RED_E_EX] + st->red[RED_E_AN] + st->red[RED_E_ZEE] + st->red[RED_E_DMI] +
                  st->red[RED_E_DEMAG];
    } else if (req_done == REQ_TORQUE) {
        R.value = torque_from(R.t_metric, st->red[RED_TMAX], st->red[RED_TSUM], st->red[RED_TSUM2], R.n_cells);
    }

    // --- run the program until it issues the next request or finishes ---
    for (int guard = 0; guard < 64; ++guard) {
        // inside advance(): keep stepping until the target is reached (advance_accepted, relax.rs:247-272)
        if (R.adv_active) {
            if (R.accepted >= R.adv_target) {
                R.adv_active = 0;
                R.pc = R.ret_pc;
            } else if (R.accepted >= S.max_acc) {
                R.adv_active = 0;
                R.pc = R.adv_fail_pc;
            } else {
                st->max_err = R.max_err;
                st->headroom = S.headroom;
                st->dt_min = S.dt_min;
                st->dt_max = S.dt_max;
                st->attempts_left = -1;
                st->target_acc = -1;
                st->req = REQ_STEP;
                return;
            }
        }
        switch (R.pc) {
            case RP_START:
                if (S.phase1) {
                    st->req = REQ_ENERGY;
                    R.pc = RP_P1_E0;
                    return;
                }
                R.pc = RP_P2_START;
                break;
            case RP_P1_E0:
                R.e0 = R.value;
                R.adv_active = 1;
                R.adv_target = R.accepted + (S.energy_stride > 1 ? S.energy_stride : 1);
                R.ret_pc = RP_P1_ADV;
                R.adv_fail_pc = RP_FAIL_P1;
                break;
            case RP_P1_ADV:
                st->req = REQ_ENERGY;
                R.pc = RP_P1_E1;
                return;
            case RP_P1_E1: {
                const double tol = S.rel_energy_tol * fmax(fabs(R.e0), 1e-30);
                if (R.value < R.e0 - tol) {
                    R.e0 = R.value;
                    R.adv_active = 1;
                    R.adv_target = R.accepted + (S.energy_stride > 1 ? S.energy_stride : 1);
                    R.ret_pc = RP_P1_ADV;
                    R.adv_fail_pc = RP_FAIL_P1;
                } else {
                    R.pc = RP_P2_START;
                }
                break;
            }
            case RP_P2_START:
                if (!S.phase2) {
                    R.has_ft = 0;
                    R.has_ftm = 0;
                    R.stop_reason = 1;  // Phase2Disabled
                    R.pc = RP_DONE;
                    break;
                }
                // torque_now(metric) -> RP_STAGE_T0
                R.checks += 1;
                R.t_metric = S.metric;
                if (R.last_b_eff_valid) {
                    R.value = torque_from(S.metric, R.tcache_max, R.tcache_sum, R.tcache_sum2, R.n_cells);
                    R.pc = RP_STAGE_T0;
                } else {
                    R.rebuilds += 1;
                    st->req = REQ_TORQUE;
                    R.pc = RP_STAGE_T0;
                    return;
                }
                break;
            case RP_STAGE_T0: {
                R.t_prev = R.value;
                const bool plateau = !S.has_thr && S.plateau_checks > 0;
                const long long pmin = S.plateau_min_checks > 1 ? S.plateau_min_checks : 1;
                R.f32mode = plateau && S.metric == 3 && S.plateau_rel == 0.0 && S.plateau_abs == 0.0 &&
                            S.plateau_checks == 1 && pmin == 1;
                R.t_prev_f32 = R.f32mode ? (float)(R.t_prev * R.n_cells) : (float)R.t_prev;
                R.fails = 0;
                R.comparisons = 0;
                R.pc = RP_STAGE_LOOP;
                break;
            }
            case RP_STAGE_LOOP: {
                const bool plateau = !S.has_thr && S.plateau_checks > 0;
                const long long need = S.plateau_checks > 1 ? S.plateau_checks : 1;
                if (S.has_thr && R.t_prev <= S.thr) {
                    R.last_stage = 0;  // BelowThreshold
                    R.pc = RP_STAGE_END;
                    break;
                }
                if (plateau && R.fails >= need) {
                    R.last_stage = 1;  // Plateau
                    R.pc = RP_STAGE_END;
                    break;
                }
                if (R.accepted >= S.max_acc) {
                    R.last_stage = 2;
                    R.has_ft = 1;
                    R.ft = R.t_prev;
                    R.stop_reason = 0;
                    R.pc = RP_DONE;
                    break;
                }
                R.adv_active = 1;
                R.adv_target = R.accepted + (S.check_stride > 1 ? S.check_stride : 1);
                R.ret_pc = RP_STAGE_ADV;
                R.adv_fail_pc = RP_FAIL_STAGE;
                break;
            }
            case RP_STAGE_ADV:
                R.checks += 1;
                R.t_metric = S.metric;
                if (R.last_b_eff_valid) {
                    R.value = torque_from(S.metric, R.tcache_max, R.tcache_sum, R.tcache_sum2, R.n_cells);
                    R.pc = RP_STAGE_TNEW;
                } else {
                    R.rebuilds += 1;
                    st->req = REQ_TORQUE;
                    R.pc = RP_STAGE_TNEW;
                    return;
                }
                break;
            case RP_STAGE_TNEW: {
                const double t_new = R.value;
                const bool plateau = !S.has_thr && S.plateau_checks > 0;
                const long long pmin = S.plateau_min_checks > 1 ? S.plateau_min_checks : 1;
                if (plateau) {
                    R.comparisons += 1;
                    if (R.comparisons < pmin) {
                        R.fails = 0;
                    } else if (R.f32mode) {
                        const float tn = (float)(t_new * R.n_cells);
                        const bool improved = tn < R.t_prev_f32;
                        R.t_prev_f32 = tn;
                        R.fails = improved ? 0 : R.fails + 1;
                    } else {
                        const double needv = fmax(S.plateau_rel * fmax(fabs(R.t_prev), 1e-30), S.plateau_abs);
                        R.fails = (R.t_prev - t_new) > needv ? 0 : R.fails + 1;
                    }
                }
                R.t_prev = t_new;
                R.pc = RP_STAGE_LOOP;
                break;
            }
            case RP_STAGE_END:
                R.has_ft = 1;
                R.ft = R.t_prev;
                if (R.max_err <= S.tighten_floor) {
                    // final max torque
                    R.checks += 1;
                    R.t_metric = 0;
                    if (R.last_b_eff_valid) {
                        R.value = R.tcache_max;
                        R.pc = RP_FINAL_T;
                    } else {
                        R.rebuilds += 1;
                        st->req = REQ_TORQUE;
                        R.pc = RP_FINAL_T;
                        return;
                    }
                } else {
                    R.max_err *= S.tighten_factor;
                    if (R.max_err < S.tighten_floor) R.max_err = S.tighten_floor;
                    R.pc = RP_P2_START;
                }
                break;
            case RP_FINAL_T:
                R.ftm = R.value;
                R.has_ftm = 1;
                if ((S.has_gate || S.has_gmax) && S.gate_extra > 0) {
                    R.gate_start = R.accepted;
                    R.gate_last_t = R.has_ft ? R.ft : INFINITY;
                    R.gfails = 0;
                    R.pc = RP_GATE_LOOP;
                } else {
                    R.stop_reason = 2;  // TightenFloorReached
                    R.pc = RP_DONE;
                }
                break;
            case RP_GATE_LOOP:
                R.checks += 1;
                R.t_metric = S.metric;
                if (R.last_b_eff_valid) {
                    R.value = torque_from(S.metric, R.tcache_max, R.tcache_sum, R.tcache_sum2, R.n_cells);
                    R.pc = RP_GATE_TMETRIC;
                } else {
                    R.rebuilds += 1;
                    st->req = REQ_TORQUE;
                    R.pc = RP_GATE_TMETRIC;
                    return;
                }
                break;
            case RP_GATE_TMETRIC:
                R.t_metric_v = R.value;
                R.t_max_v = NAN;
                if (S.has_gmax || S.metric == 0) {
                    if (S.metric == 0) {
                        R.t_max_v = R.t_metric_v;
                    } else {
                        R.checks += 1;
                        R.t_metric = 0;
                        if (R.last_b_eff_valid) {
                            R.t_max_v = R.tcache_max;
                        } else {
                            R.rebuilds += 1;
                            st->req = REQ_TORQUE;
                            R.pc = RP_GATE_TMAX;
                            return;
                        }
                    }
                }
                R.pc = RP_GATE_TMAX;
                R.value = R.t_max_v;
                break;
            case RP_GATE_TMAX: {
                R.t_max_v = R.value;
                const bool okm = !S.has_gate || R.t_metric_v <= S.gate;
                const bool okx = !S.has_gmax || R.t_max_v <= S.gate_max;
                R.has_ft = 1;
                R.ft = R.t_metric_v;
                if (std::isfinite(R.t_max_v)) {
                    R.has_ftm = 1;
                    R.ftm = R.t_max_v;
                }
                if (okm && okx) {
                    R.stop_reason = 2;
                    R.pc = RP_DONE;
                    break;
                }
                if (R.accepted - R.gate_start >= S.gate_extra) {
                    R.stop_reason = 3;  // TorqueGateNotSatisfied
                    R.pc = RP_DONE;
                    break;
                }
                if (S.gate_plateau_fails > 0) {
                    const double needv = fmax(S.plateau_rel * fmax(fabs(R.gate_last_t), 1e-30), S.plateau_abs);
                    R.gfails = (R.gate_last_t - R.t_metric_v) > needv ? 0 : R.gfails + 1;
                    if (R.gfails >= S.gate_plateau_fails) {
                        R.stop_reason = 3;
                        R.pc = RP_DONE;
                        break;
                    }
                    R.gate_last_t = R.t_metric_v;
                }
                R.adv_active = 1;
                R.adv_target = R.accepted + (S.check_stride > 1 ? S.check_stride : 1);
                R.ret_pc = RP_GATE_LOOP;
                R.adv_fail_pc = RP_FAIL_GATE;
                break;
            }
            case RP_FAIL_P1:  // advance() failed in phase 1 (relax.rs:402-425)
                R.stop_reason = 0;
                R.pc = RP_DONE;
                break;
            case RP_FAIL_STAGE:  // advance() failed inside a stage (relax.rs:531-546)
                R.last_stage = 2;
                R.has_ft = 1;
                R.ft = R.t_prev;
                R.stop_reason = 0;
                R.pc = RP_DONE;
                break;
            case RP_FAIL_GATE:  // advance() failed in the gate loop (relax.rs:720-736)
                R.last_stage = 2;
                R.stop_reason = 0;
                R.pc = RP_DONE;
                break;
            case RP_DONE:
            default:
                R.done = 1;
                st->active = 0;
                return;
        }
    }
}

#ifdef __CUDACC__
__global__ void k_relax_control(FilmDev* films, RelaxStateDev* rs_all, int nfilms, RelaxSettingsDev S) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfilms) return;
    relax_control_core(films[f].st, rs_all[f], S);
}
#endif

}  // namespace llg
