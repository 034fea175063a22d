"""Generate the FP64 oracle record of the 128x32 relax-then-field flow.

Relax (relax_with_report, relax.rs:334) from the Gaussian-tilt state, then 1 ns
of RK45 under 20 mT in 10 ps windows with dt clamped onto each window end
(st_problems/sp4.rs:306-333).  Writes film_128x32_flow.npz next to this file:
the relax report, the relaxed m, per-window accepted/rejected counts and <m>,
and the final m.  Takes about half an hour on 8 host threads.

    python tests/golden/make_film_128x32_flow.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "llg-sim_b200"))
import oracle as orc  # noqa: E402
import workloads as W  # noqa: E402

REPORT_FIELDS = ["accepted_steps", "rejected_steps", "torque_checks", "torque_field_rebuilds", "stop_reason",
                 "last_stage_stop", "final_torque", "final_torque_max", "final_max_err", "final_dt"]


def main():
    f, rx, run = W.film_128x32_relax_then_field()
    g = orc.make_grid(f.nx, f.ny, f.dx, f.dy, f.dz)
    mat = orc.make_material(f.ms, f.a_ex, f.k_u, f.easy, f.dmi, f.demag)
    S = orc.Solver(g, mat)
    m = f.m0.copy()
    p = orc.make_params(W.GAMMA, rx["alpha"], rx["dt0"], (0.0, 0.0, 0.0))
    st = orc.default_relax_settings(**{k: v for k, v in rx.items() if k not in ("alpha", "dt0")})
    t0 = time.time()
    rep = S.relax(m, p, orc.FIELD_FULL, st)
    print("relax", rep.stop_reason, rep.accepted_steps, rep.rejected_steps, rep.final_torque_max,
          f"{time.time() - t0:.1f}s", flush=True)
    m_relaxed = m.copy()
    relax_dt = p.dt
    p = orc.make_params(W.GAMMA, run["alpha"], run["dt0"], f.b_ext)
    n_out = int(round(run["t_total"] / run["dt_out"]))
    acc = np.zeros(n_out, dtype=np.int64)
    rej = np.zeros(n_out, dtype=np.int64)
    mean = np.zeros((n_out, 3))
    for k in range(n_out):
        t = 0.0
        while t + 1e-18 < run["dt_out"]:
            rem = run["dt_out"] - t
            if p.dt > rem:
                p.dt = rem
            _, a, dtu = S.step_rk45(m, p, orc.FIELD_FULL, run["max_err"], run["headroom"], run["dt_min"],
                                    run["dt_max"])
            if a:
                t += dtu
                acc[k] += 1
            else:
                rej[k] += 1
        mean[k] = m.mean(axis=0)
    print("run", acc.sum(), rej.sum(), mean[-1], f"{time.time() - t0:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, "film_128x32_flow.npz"), m0=f.m0, m_relaxed=m_relaxed, m_final=m,
                        relax=np.array([float(getattr(rep, k)) for k in REPORT_FIELDS]), relax_max_err=st.max_err,
                        relax_dt=np.float64(relax_dt), window_acc=acc, window_rej=rej, window_mean=mean)


if __name__ == "__main__":
    main()
