"""The device-resident minimiser (minimize_damping_only, minimize.rs:107) and
the gated relax policy (relax_until_gate, equilibrate.rs:159) on the GPU,
against the FP64 oracle."""
import numpy as np
import pytest

import equilibrate as E
from helpers import GAMMA, case, gpu_solver, holes_mask, oracle_solver

pytestmark = pytest.mark.gpu

# (name, nx, ny, init, seed, field mask, b_ext, material extras, holes, settings overrides)
CASES = [
    ("threshold", 16, 12, "noise", 4, 2, (0.05, 0.0, 0.0), {}, None, dict(max_iters=5000)),
    ("dm_stop", 16, 12, "noise", 4, 2, (0.05, 0.0, 0.0), {}, None,
     dict(max_iters=5000, torque_threshold=1e-6, dm_stop=1e-5)),
    ("stall", 16, 12, "random", 4, 2, (0.01, 0.0, 0.0), {}, None,
     dict(max_iters=5000, dm_stop=None, min_iters_before_stall=100, stall_iters=50)),
    ("max_iters", 16, 12, "random", 4, 2, (0.01, 0.0, 0.0), {}, None, dict(max_iters=40, dm_stop=None)),
    ("holes_dmi", 32, 32, "noise", 7, 2, (0.05, 0.0, 0.0), dict(dmi=1e-3), [(4, 2, 6)], dict(max_iters=5000)),
    ("local_only", 32, 32, "noise", 7, 1, (0.05, 0.0, 0.0), dict(dmi=1e-3), [(4, 2, 6)], dict(max_iters=5000)),
    ("film_128x64", 128, 64, "noise", 9, 2, (0.02, 0.01, 0.0), {}, None, dict(max_iters=3000)),
]


def _init(orc, n, init, seed, mask):
    m = orc.init_uniform_with_noise(n, (1.0, 0.0, 0.0), 0.2, seed) if init == "noise" else orc.init_random(n, seed)
    if mask is not None:
        m[mask == 0] = 0.0
    return m


def _exit(r):
    return (int(r.converged), int(r.stalled), int(r.dm_converged))


@pytest.mark.parametrize("name,nx,ny,init,seed,fmask,bext,extra,holes,kw", CASES, ids=[c[0] for c in CASES])
def test_minimize_fp64_matches_oracle(orc, gpu, name, nx, ny, init, seed, fmask, bext, extra, holes, kw):
    mask = holes_mask(nx, ny, holes) if holes else None
    c = case(nx, ny, mask=mask, **extra)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, gpu.FP64)
    m0 = _init(orc, nx * ny, init, seed, mask)
    g.set_state(m0)
    mo = m0.copy()
    ro = o.minimize(mo, orc.make_params(GAMMA, 0.5, 1e-13, bext), fmask, orc.default_minimize_settings(**kw))
    n0 = g.launch_count()
    rg = g.minimize(gpu.LLGParams(GAMMA, 0.5, 1e-13, bext), fmask, gpu.MinimizeSettings.default(**kw))
    assert g.launch_count() > n0
    # FP64 with the GPU's FFT and fused multiply-adds: the same decisions, values to round-off
    assert _exit(rg) == _exit(ro)
    assert rg.iters == ro.iters
    assert rg.final_lambda == pytest.approx(ro.final_lambda, rel=1e-12)
    for f in ("final_torque", "final_tmean"):
        assert getattr(rg, f) == pytest.approx(getattr(ro, f), rel=1e-7, abs=1e-12), f
    assert rg.final_max_dm == pytest.approx(ro.final_max_dm, rel=1e-6, abs=1e-13)
    mg = g.get_state()
    assert np.abs(mg - mo).max() < 1e-9
    if mask is not None:
        assert not mg[mask == 0].any()


def test_minimize_max_iters_zero(gpu):
    c = case(16, 12)
    g = gpu_solver(gpu, c, gpu.FP32)
    m = np.tile([1.0, 0.0, 0.0], (16 * 12, 1))
    g.set_state(m)
    r = g.minimize(gpu.LLGParams(GAMMA, 0.5, 1e-13), 2, gpu.MinimizeSettings.default(max_iters=0))
    assert r.iters == 0 and np.isinf(r.final_torque) and np.isinf(r.final_max_dm) and np.isinf(r.final_tmean)
    assert r.final_lambda == 2e-2
    assert np.array_equal(g.get_state(), m)


def test_minimize_fp32_reaches_threshold(orc, gpu):
    """FP32 state storage rounds every update, so the descent path differs from the
    FP64 oracle's by round-off; the FP32 result is checked as a minimised state:
    the FP64 oracle sees max torque below the threshold at the GPU's final m
    (FP32 field allowance 2 %), in the same minimum as the oracle's result."""
    nx, ny, bext = 64, 32, (0.05, 0.0, 0.0)
    c = case(nx, ny)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, gpu.FP32)
    m0 = _init(orc, nx * ny, "noise", 21, None)
    g.set_state(m0)
    mo = m0.copy()
    kw = dict(max_iters=5000, torque_threshold=5e-4)
    ro = o.minimize(mo, orc.make_params(GAMMA, 0.5, 1e-13, bext), 2, orc.default_minimize_settings(**kw))
    rg = g.minimize(gpu.LLGParams(GAMMA, 0.5, 1e-13, bext), 2, gpu.MinimizeSettings.default(**kw))
    assert rg.converged and ro.converged
    assert abs(rg.iters - ro.iters) <= max(5, ro.iters // 20)
    mg = g.get_state()
    b = o.build_h_eff(mg, bext)
    assert orc.torque_metric(mg, b, orc.TORQUE_MAX) <= 5e-4 * 1.02
    assert np.abs(mg - mo).max() < 1e-3


def test_batch_minimize_equals_single_films(orc, gpu):
    """Films of different sizes and materials minimised together: each film's
    report and state equal its own FP64 oracle run."""
    specs = [(16, 12, 4, (0.05, 0.0, 0.0), {}), (32, 16, 5, (0.0, 0.04, 0.0), dict(ms=6e5)),
             (24, 24, 6, (0.03, 0.03, 0.0), dict(a_ex=1.0e-11))]
    kw = dict(max_iters=4000)
    grids, mats, params, oracle_runs, m0s = [], [], [], [], []
    for nx, ny, seed, bext, extra in specs:
        c = case(nx, ny, **extra)
        grids.append(gpu.Grid2D(c["nx"], c["ny"], c["dx"], c["dy"], c["dz"]))
        mats.append(gpu.Material(c["ms"], c["a_ex"], c["k_u"], c["easy"], c["dmi"], c["demag"]))
        params.append(gpu.LLGParams(GAMMA, 0.5, 1e-13, bext))
        m0 = _init(orc, nx * ny, "noise", seed, None)
        m0s.append(m0)
        mo = m0.copy()
        ro = oracle_solver(orc, c).minimize(mo, orc.make_params(GAMMA, 0.5, 1e-13, bext), 2,
                                            orc.default_minimize_settings(**kw))
        oracle_runs.append((ro, mo))
    b = gpu.Batch(grids, mats, gpu.FP64)
    for f, m0 in enumerate(m0s):
        b.set_state(f, m0)
    reps = b.minimize(params, 2, gpu.MinimizeSettings.default(**kw))
    for f, (ro, mo) in enumerate(oracle_runs):
        assert reps[f].iters == ro.iters, f
        assert _exit(reps[f]) == _exit(ro)
        assert reps[f].final_torque == pytest.approx(ro.final_torque, rel=1e-7)
        assert np.abs(b.get_state(f) - mo).max() < 1e-9


def test_minimize_invalidates_fsal_and_steps_continue(orc, gpu):
    """An RK45 step after a minimiser pass starts from the minimised state (the
    FSAL torque of the earlier state is dropped)."""
    nx, ny, bext = 16, 12, (0.05, 0.0, 0.0)
    c = case(nx, ny)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, gpu.FP64)
    m0 = _init(orc, nx * ny, "noise", 4, None)
    g.set_state(m0)
    pg = gpu.LLGParams(GAMMA, 0.5, 1e-13, bext)
    g.step_rk45(pg, 2, 1e-5, 0.8, 1e-18, 1e-11)   # leaves a valid FSAL torque behind
    mo = g.get_state()
    g.minimize(pg, 2, gpu.MinimizeSettings.default(max_iters=30, dm_stop=None))
    o.minimize(mo, orc.make_params(GAMMA, 0.5, 1e-13, bext), 2,
               orc.default_minimize_settings(max_iters=30, dm_stop=None))
    po = orc.make_params(GAMMA, 0.5, pg.dt, bext)
    o.invalidate()
    eo, ao, _ = o.step_rk45(mo, po, 2, 1e-5, 0.8, 1e-18, 1e-11)
    eg, ag, _ = g.step_rk45(pg, 2, 1e-5, 0.8, 1e-18, 1e-11)
    assert ag == ao
    assert eg == pytest.approx(eo, rel=1e-6)
    assert np.abs(g.get_state() - mo).max() < 1e-9


def test_relax_until_gate_matches_oracle(orc, gpu):
    """The gated relax policy driving the GPU solver and the oracle: the same
    passes, minimiser fallbacks and gate outcome."""
    nx, ny, bext = 16, 12, (0.05, 0.0, 0.0)
    c = case(nx, ny)

    class OracleSolver:
        def __init__(self, s, m):
            self.s, self.m = s, m

        def relax(self, params, fmask, st):
            return self.s.relax(self.m, params, fmask, st)

        def minimize(self, params, fmask, st):
            return self.s.minimize(self.m, params, fmask, st)

        def torque_metric(self, params, fmask, metric):
            return orc.torque_metric(self.m, self.s.build_h_eff(self.m, tuple(params.b_ext), fmask), metric)

    m0 = _init(orc, nx * ny, "noise", 4, None)
    rkw = dict(torque_threshold=None, torque_metric=1, torque_plateau_checks=8, torque_plateau_min_checks=8,
               torque_plateau_rel=0.0, torque_plateau_abs=1e-7, max_err=1e-5, max_accepted_steps=400)
    mkw = dict(max_iters=50, torque_threshold=8e-4)
    osv = OracleSolver(oracle_solver(orc, c), m0.copy())
    out_o = E.relax_until_gate(osv, orc.make_params(GAMMA, 0.5, 1e-13, bext), 2, orc.default_relax_settings(**rkw),
                               E.RelaxGate(torque_gate=1e-9, extra_passes=2, fallback_to_minimize=True,
                                           minimize=orc.default_minimize_settings(**mkw)))
    g = gpu_solver(gpu, c, gpu.FP64)
    g.set_state(m0)
    out_g = E.relax_until_gate(g, gpu.LLGParams(GAMMA, 0.5, 1e-13, bext), 2, gpu.RelaxSettings.default(**rkw),
                               E.RelaxGate(torque_gate=1e-9, extra_passes=2, fallback_to_minimize=True,
                                           minimize=gpu.MinimizeSettings.default(**mkw)))
    assert out_g.gate_passed == out_o.gate_passed
    assert len(out_g.relax_passes) == len(out_o.relax_passes)
    assert len(out_g.minimize_passes) == len(out_o.minimize_passes)
    for a, b in zip(out_g.relax_passes, out_o.relax_passes):
        assert a.stop_reason == b.stop_reason
        assert a.final_torque_max == pytest.approx(b.final_torque_max, rel=0.05)
    assert np.abs(g.get_state() - osv.m).max() < 1e-3
