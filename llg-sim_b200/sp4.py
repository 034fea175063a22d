"""The µMAG standard problem 4 driver flow (st_problems/sp4.rs:140-370) on the GPU.

A 500 x 125 x 3 nm Permalloy film (200 x 50 cells, Ms 8e5 A/m, A 13e-12 J/m,
no anisotropy, demag on) starts uniform along normalize(1, 0.1, 0), relaxes
with the reference's SP4 relax settings (RK23 with the energy and torque
phases, max |m x B| 1e-4 T, tightening to 1e-9), then runs 1 ns of RK45
(max_err 1e-5, alpha 0.02, dt 1e-13 in [1e-19, 1e-11]) under field a
(-24.6, 4.3, 0) mT or b (-35.5, -6.3, 0) mT, landing on every 10 ps sample.
Outputs as the reference writes them: table.csv (t_s,mx,my,mz in {:.16e}),
text OVF snapshots m0000000.ovf .. every 100 ps, and m_mx_zero.ovf at the
first sample where <mx> crosses from > 0 to <= 0.

The relax runs as one device-resident llg_relax call; each 10 ps sample is one
device-resident llg_run_rk45 call with t_end clamped onto the sample time (the
reference's per-step clamp, sp4.rs:306-333).
"""
import math
import os

import numpy as np

import llg_b200 as L

FIELDS = {"a": (-24.6e-3, 4.3e-3, 0.0), "b": (-35.5e-3, -6.3e-3, 0.0)}


def sp4_setup():
    nx, ny = 200, 50
    grid = L.Grid2D(nx, ny, 500e-9 / nx, 125e-9 / ny, 3e-9)
    mat = L.Material(8.0e5, 13e-12, 0.0, (0.0, 0.0, 1.0), None, True)
    return grid, mat


def sp4_relax_settings():
    """sp4.rs:210-236: RelaxSettings with the SP4 overrides, the rest default."""
    return L.RelaxSettings.default(max_err=1e-5, headroom=0.8, dt_min=1e-18, dt_max=1e-11, phase1_enabled=1,
                                   phase2_enabled=1, energy_stride=3, rel_energy_tol=1e-12,
                                   torque_metric=L.TORQUE_MAX, torque_threshold=1e-4, torque_check_stride=1,
                                   tighten_factor=1.0 / math.sqrt(2.0), tighten_floor=1e-9,
                                   max_accepted_steps=2000000, torque_plateau_checks=0)


def _fmt(v):
    return L.rust_exp(v, 16)


def run_sp4(case="a", out_dir=None, precision=L.FP64, t_total=1e-9, dt_out=10e-12, dt_ovf=100e-12, device=0,
            log=print, solver=None):
    """Runs SP4 case 'a' or 'b'; returns a summary dict.  out_dir defaults to the
    reference's runs/st_problems/sp4/sp4{a,b}_rust.  `solver` replaces the GPU solver
    of the 200x50 film (an object with the llg_b200.Solver methods used here)."""
    case = case.lower()
    b_ext = FIELDS.get(case, FIELDS["a"])
    if out_dir is None:
        out_dir = os.path.join("runs", "st_problems", "sp4", f"sp4{case if case in FIELDS else 'a'}_rust")
    os.makedirs(out_dir, exist_ok=True)
    grid, mat = sp4_setup()
    s = solver if solver is not None else L.Solver(grid, mat, precision, device=device)
    m0 = np.array([1.0, 0.1, 0.0]) / math.sqrt(1.01)
    s.set_state(np.tile(m0, (grid.nx * grid.ny, 1)))

    # relax stage, B_ext = 0 (sp4.rs:198-265)
    p_relax = L.LLGParams(L.GAMMA_E_RAD_PER_S_T, 0.02, 5e-14, (0.0, 0.0, 0.0))
    t0 = s.torque_metric(p_relax, L.FULL, L.TORQUE_MAX)
    st = sp4_relax_settings()
    rep = s.relax(p_relax, L.FULL, st)
    t1 = s.torque_metric(p_relax, L.FULL, L.TORQUE_MAX)
    log(f"SP4{case.upper()} relax: start |m x B|_inf = {L.rust_exp(t0, 3)}, done {L.rust_exp(t1, 3)}, "
        f"final max_err={L.rust_exp(st.max_err, 3)}, final dt={L.rust_exp(p_relax.dt, 3)}")

    # run stage (sp4.rs:267-360)
    p = L.LLGParams(L.GAMMA_E_RAD_PER_S_T, 0.02, 1e-13, b_ext)
    dt_min, dt_max = 1e-13 * 1e-6, 1e-13 * 100.0
    n_out = int(round(t_total / dt_out))
    stride = int(round(dt_ovf / dt_out))
    rows = []
    mx, my, mz = s.mean_m()
    rows.append((0.0, mx, my, mz))
    prev_mx = mx
    snap = 0

    def snapshot(name, t):
        s.write_ovf2(os.path.join(out_dir, name), L.OvfMeta.magnetization().with_total_sim_time(t), L.OVF_TEXT)

    snapshot(f"m{snap:07d}.ovf", 0.0)
    snap += 1
    crossover = None
    accepted = rejected = 0
    for k in range(1, n_out + 1):
        t_target = k * dt_out
        a, r, _ = s.run_rk45(p, L.FULL, 1e-5, 0.8, dt_min, dt_max, t_end=t_target - (k - 1) * dt_out,
                             max_attempts=50_000_000)
        accepted += a
        rejected += r
        mx, my, mz = s.mean_m()
        rows.append((t_target, mx, my, mz))
        if crossover is None and prev_mx > 0.0 and mx <= 0.0:
            snapshot("m_mx_zero.ovf", t_target)
            crossover = t_target
            log(f"SP4{case.upper()} wrote mx=0 crossover OVF at t={L.rust_exp(t_target, 6)} s")
        prev_mx = mx
        if stride > 0 and k % stride == 0:
            snapshot(f"m{snap:07d}.ovf", t_target)
            snap += 1
    with open(os.path.join(out_dir, "table.csv"), "w") as f:
        f.write("t_s,mx,my,mz\n")
        for row in rows:
            f.write(",".join(_fmt(v) for v in row) + "\n")
    s.close()
    return {"relax_accepted": rep.accepted_steps, "relax_torque": t1, "run_accepted": int(accepted),
            "run_rejected": int(rejected), "snapshots": snap, "crossover_t": crossover, "rows": rows,
            "out_dir": out_dir}


if __name__ == "__main__":
    import sys

    c = sys.argv[1] if len(sys.argv) > 1 else "a"
    out = run_sp4(c)
    print(f"SP4{c.upper()} wrote {os.path.join(out['out_dir'], 'table.csv')} and {out['snapshots']} OVF snapshots")
