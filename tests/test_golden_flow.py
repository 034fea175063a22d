"""The 128x32 flow fixture is the oracle's own record: its first 10 ps windows
re-run on the CPU from the stored relaxed state reproduce the stored <m>."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "llg-sim_b200"))
import workloads as W  # noqa: E402


def test_flow_fixture_windows_reproduce(orc):
    g = np.load(os.path.join(HERE, "golden", "film_128x32_flow.npz"))
    f, rx, run = W.film_128x32_relax_then_field()
    assert np.array_equal(g["m0"], f.m0)
    S = orc.Solver(orc.make_grid(f.nx, f.ny, f.dx, f.dy, f.dz),
                   orc.make_material(f.ms, f.a_ex, f.k_u, f.easy, f.dmi, f.demag))
    m = g["m_relaxed"].copy()
    p = orc.make_params(W.GAMMA, run["alpha"], run["dt0"], f.b_ext)
    for k in range(2):
        t, acc = 0.0, 0
        while t + 1e-18 < run["dt_out"]:
            p.dt = min(p.dt, run["dt_out"] - t)
            _, a, dtu = S.step_rk45(m, p, orc.FIELD_FULL, run["max_err"], run["headroom"], run["dt_min"],
                                    run["dt_max"])
            if a:
                t += dtu
                acc += 1
        assert acc == g["window_acc"][k]
        assert np.abs(m.mean(axis=0) - g["window_mean"][k]).max() < 1e-13
