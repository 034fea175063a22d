"""End-to-end flow on the 128x32 film: relax, then 1 ns of RK45 under 20 mT with
<m> sampled every 10 ps (the reference's SP4 driver flow, st_problems/sp4.rs:
198-333), against the FP64 oracle's record in tests/golden/film_128x32_flow.npz
(made by tests/golden/make_film_128x32_flow.py)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "llg-sim_b200"))
import workloads as W  # noqa: E402

pytestmark = pytest.mark.gpu
REPORT = ["accepted_steps", "rejected_steps", "torque_checks", "torque_field_rebuilds", "stop_reason",
          "last_stage_stop", "final_torque", "final_torque_max", "final_max_err", "final_dt"]


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "film_128x32_flow.npz"))


def _solver(gpu, prec):
    f, rx, run = W.film_128x32_relax_then_field()
    return f, rx, run, gpu.Solver(f.grid(gpu), f.material(gpu), prec)


def _run_windows(gpu, S, f, run):
    p = gpu.LLGParams(W.GAMMA, run["alpha"], run["dt0"], f.b_ext)
    n_out = int(round(run["t_total"] / run["dt_out"]))
    acc = np.zeros(n_out, dtype=np.int64)
    rej = np.zeros(n_out, dtype=np.int64)
    mean = np.zeros((n_out, 3))
    for k in range(n_out):
        a, r, t = S.run_rk45(p, gpu.FULL, run["max_err"], run["headroom"], run["dt_min"], run["dt_max"],
                             t_end=run["dt_out"])
        assert t == pytest.approx(run["dt_out"], rel=1e-12)
        acc[k], rej[k] = a, r
        mean[k] = S.mean_m()
    return acc, rej, mean


@pytest.mark.parametrize("prec", [1, 0])
def test_relax_phase_matches_oracle(gpu, golden, prec):
    f, rx, run, S = _solver(gpu, prec)
    S.set_state(golden["m0"])
    p = gpu.LLGParams(W.GAMMA, rx["alpha"], rx["dt0"], (0.0, 0.0, 0.0))
    st = gpu.RelaxSettings.default(**{k: v for k, v in rx.items() if k not in ("alpha", "dt0")})
    rep = S.relax(p, gpu.FULL, st)
    ref = dict(zip(REPORT, golden["relax"]))
    assert rep.stop_reason == int(ref["stop_reason"]) == 2
    assert rep.final_torque_max <= rx["torque_threshold"]
    mg = S.get_state()
    if prec == 1:
        # tens of thousands of FP64 steps: counts agree to round-off-level decision flips
        assert abs(rep.accepted_steps - ref["accepted_steps"]) <= 0.02 * ref["accepted_steps"]
        assert np.abs(mg - golden["m_relaxed"]).max() < 1e-3
    else:
        assert np.abs(mg.mean(axis=0) - golden["m_relaxed"].mean(axis=0)).max() < 1e-3


@pytest.mark.parametrize("prec,tol", [(1, 1e-8), (0, 1e-4)])
def test_field_run_matches_oracle(gpu, golden, prec, tol):
    """1 ns under 20 mT from the oracle's relaxed state: <m> every 10 ps within tol of FP64."""
    f, rx, run, S = _solver(gpu, prec)
    S.set_state(golden["m_relaxed"])
    acc, rej, mean = _run_windows(gpu, S, f, run)
    assert np.abs(mean - golden["window_mean"]).max() < tol
    if prec == 1:
        assert np.abs(acc - golden["window_acc"]).max() <= 1
        assert abs(int(acc.sum()) - int(golden["window_acc"].sum())) <= 3
        assert np.abs(S.get_state() - golden["m_final"]).max() < 1e-7
