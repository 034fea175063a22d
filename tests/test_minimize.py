"""CPU tests of the minimiser and the gated relax policy.

* The oracle's minimize_damping_only restatement (minimize.rs:107-369) against a
  second, pure-Python restatement of the same loop on the oracle's field.
* The device minimiser controller (minimize_control_core in minimize_dev.cuh),
  compiled for the host and driven by the oracle's field builder, against the
  oracle: every report field and the final state must be equal, for every way
  the loop can end (threshold, dM stop with and without its torque gates,
  stall, max_iters, max_iters = 0) and for masked films.
* relax_until_gate (equilibrate.rs:159-255) as composed in equilibrate.py,
  against a scripted solver that records the settings of every pass, and once
  end to end on the oracle."""
import ctypes as C
import math
import os
import subprocess

import numpy as np
import pytest

import equilibrate as E
from helpers import GAMMA, case, holes_mask

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REPORT = ["iters", "converged", "stalled", "dm_converged", "final_torque", "final_max_dm", "final_tmean",
          "final_lambda"]


@pytest.fixture(scope="module")
def harness(orc, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("mharness") / "libmharness.so")
    odir = os.path.join(ROOT, "oracle")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-I/usr/local/cuda/include",
                    os.path.join(HERE, "harness", "minimize_harness.cpp"), "-o", out, "-L", odir, "-loracle",
                    "-Wl,-rpath," + odir], check=True)
    H = C.CDLL(out)
    dp = C.POINTER(C.c_double)
    H.harness_minimize.argtypes = [C.POINTER(orc.Grid), C.POINTER(orc.Material), C.c_void_p, dp,
                                   C.POINTER(orc.Params), C.c_int, C.POINTER(orc.MinimizeSettings),
                                   C.POINTER(orc.MinimizeReport)]
    return H


def _setup(orc, nx, ny, init, seed, dmi=None, k_u=0.0, holes=None, bext=(0.05, 0.0, 0.0)):
    mask = holes_mask(nx, ny, holes) if holes else None
    c = case(nx, ny, dmi=dmi, k_u=k_u, mask=mask)
    g = orc.make_grid(c["nx"], c["ny"], c["dx"], c["dy"], c["dz"])
    mat = orc.make_material(c["ms"], c["a_ex"], c["k_u"], c["easy"], c["dmi"], c["demag"])
    if init == "noise":
        m = orc.init_uniform_with_noise(nx * ny, (1.0, 0.0, 0.0), 0.2, seed)
    else:
        m = orc.init_random(nx * ny, seed)
    if mask is not None:
        m[mask == 0] = 0.0
    p = orc.make_params(GAMMA, 0.5, 1e-13, bext)
    return g, mat, mask, m, p


# (name, grid / init, field mask, settings overrides, expected exit)
SCENARIOS = [
    ("threshold", dict(nx=16, ny=12, init="noise", seed=4), 2, dict(max_iters=5000), "converged"),
    ("dm_stop_gated_ok", dict(nx=16, ny=12, init="noise", seed=4), 2,
     dict(max_iters=5000, torque_threshold=1e-6, dm_stop=1e-5), "dm"),
    ("dm_stop_gate_fails", dict(nx=16, ny=12, init="noise", seed=4), 2,
     dict(max_iters=5000, torque_threshold=1e-9, dm_stop=1e-6, dm_torque_gate=1e-12), "dm"),
    ("stall", dict(nx=16, ny=12, init="random", seed=4, bext=(0.01, 0.0, 0.0)), 2,
     dict(max_iters=5000, dm_stop=None, min_iters_before_stall=100, stall_iters=50), "stalled"),
    ("max_iters", dict(nx=16, ny=12, init="random", seed=4, bext=(0.01, 0.0, 0.0)), 2,
     dict(max_iters=40, dm_stop=None), "max"),
    ("max_iters_zero", dict(nx=16, ny=12, init="random", seed=4), 2, dict(max_iters=0), "max"),
    ("holes_dmi_full", dict(nx=32, ny=32, init="noise", seed=7, dmi=1e-3, holes=[(4, 2, 6)]), 2,
     dict(max_iters=5000), "converged"),
    ("holes_dmi_local", dict(nx=32, ny=32, init="noise", seed=7, dmi=1e-3, holes=[(4, 2, 6)]), 1,
     dict(max_iters=5000), "converged"),
    ("anisotropy_exchange_only", dict(nx=32, ny=32, init="noise", seed=7, k_u=5e5), 0,
     dict(max_iters=3000), "max"),
    # edge settings: a one-sample dM window from the first iteration, an immediate stall
    ("dm_one_sample", dict(nx=16, ny=12, init="noise", seed=4), 2,
     dict(max_iters=5000, torque_threshold=1e-9, dm_stop=1e-5, dm_samples=1, dm_min_iters=0), "dm"),
    ("dm_samples_zero", dict(nx=16, ny=12, init="noise", seed=4), 2,
     dict(max_iters=5000, torque_threshold=1e-9, dm_stop=1e-5, dm_samples=0, dm_min_iters=0), "dm"),
    ("stall_immediately", dict(nx=16, ny=12, init="random", seed=4), 2,
     dict(max_iters=100, dm_stop=None, stall_iters=0, min_iters_before_stall=0), "stalled"),
    ("lambda_pinned", dict(nx=16, ny=12, init="noise", seed=4), 2,
     dict(max_iters=2000, lambda0=1e-2, lambda_min=1e-2, lambda_max=1e-2), "converged"),
]


def _exit(r):
    if r.converged and not r.dm_converged:
        return "converged"
    if r.dm_converged:
        return "dm"
    if r.stalled:
        return "stalled"
    return "max"


@pytest.mark.parametrize("name,geo,fmask,kw,expect", SCENARIOS, ids=[s[0] for s in SCENARIOS])
def test_device_minimize_controller_equals_oracle(orc, harness, name, geo, fmask, kw, expect):
    g, mat, mask, m0, p = _setup(orc, **geo)
    st = orc.default_minimize_settings(**kw)
    mo = m0.copy()
    ro = orc.Solver(g, mat, mask).minimize(mo, p, fmask, st)
    assert _exit(ro) == expect, (name, ro.iters)
    mh = m0.copy()
    rh = orc.MinimizeReport()
    mp = None
    if mask is not None:
        mk = np.ascontiguousarray(mask.astype(np.uint8))
        mp = mk.ctypes.data_as(C.c_void_p)
    rc = harness.harness_minimize(C.byref(g), C.byref(mat), mp, mh.ctypes.data_as(C.POINTER(C.c_double)),
                                  C.byref(p), fmask, C.byref(st), C.byref(rh))
    assert rc == 0
    for f in REPORT:
        a, b = getattr(rh, f), getattr(ro, f)
        assert a == b or (isinstance(a, float) and math.isinf(a) and math.isinf(b)), f
    assert np.array_equal(mh, mo)
    if mask is not None:
        assert not mo[mask == 0].any()


def _python_minimize(orc, solver, m, p, fmask, kw):
    """minimize.rs:138-368 restated directly in Python over the oracle's field."""
    s = dict(torque_threshold=5e-4, max_iters=20000, lambda0=2e-2, lambda_min=1e-5, lambda_max=5e-2, grow=1.05,
             shrink=0.8, stall_iters=5000, stall_rel=5e-4, min_iters_before_stall=500, dm_stop=1e-6, dm_samples=10,
             dm_torque_gate=2e-3, dm_torque_gate_max=5e-3, dm_min_iters=50)
    s.update(kw)
    lam, t_prev, stall, hist = s["lambda0"], math.inf, 0, []
    last_dm = last_tmax = last_tmean = math.inf
    n = m.shape[0]
    for it in range(s["max_iters"]):
        b = solver.build_h_eff(m, tuple(p.b_ext), fmask)
        tmax = tsum = max_dm = 0.0
        for i in range(n):
            m0 = [float(v) for v in m[i]]
            bb = [float(v) for v in b[i]]
            t = [m0[1] * bb[2] - m0[2] * bb[1], m0[2] * bb[0] - m0[0] * bb[2], m0[0] * bb[1] - m0[1] * bb[0]]
            tmag = math.sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2])
            tsum += tmag
            tmax = max(tmax, tmag)
            d = [t[1] * m0[2] - t[2] * m0[1], t[2] * m0[0] - t[0] * m0[2], t[0] * m0[1] - t[1] * m0[0]]
            x, y, z = m0[0] + lam * d[0], m0[1] + lam * d[1], m0[2] + lam * d[2]
            n2 = x * x + y * y + z * z
            if n2 > 0.0:
                inv = 1.0 / math.sqrt(n2)
                x, y, z = x * inv, y * inv, z * inv
            dx, dy, dz = x - m0[0], y - m0[1], z - m0[2]
            max_dm = max(max_dm, math.sqrt(dx * dx + dy * dy + dz * dz))
            m[i] = (x, y, z)
        tmean = tsum / max(float(n), 1.0)
        last_tmean = tmean
        if tmax < s["torque_threshold"]:
            return (it + 1, tmax, True, False, max_dm, False, tmean, lam)
        last_dm, last_tmax = max_dm, tmax
        if s["dm_stop"] is not None and it + 1 >= s["dm_min_iters"]:
            hist.append(max_dm)
            hist = hist[-max(s["dm_samples"], 1):]
            if len(hist) == max(s["dm_samples"], 1) and all(v < s["dm_stop"] for v in hist):
                ok = (s["dm_torque_gate"] is None or tmean <= s["dm_torque_gate"]) and \
                     (s["dm_torque_gate_max"] is None or tmax <= s["dm_torque_gate_max"])
                return (it + 1, tmax, ok, False, max_dm, True, tmean, lam)
        lam = min(lam * s["grow"], s["lambda_max"]) if tmean < t_prev else max(lam * s["shrink"], s["lambda_min"])
        if it + 1 >= s["min_iters_before_stall"] and math.isfinite(t_prev):
            stall = stall + 1 if (t_prev - tmean) <= s["stall_rel"] * max(abs(t_prev), 1e-30) else 0
        if stall >= s["stall_iters"]:
            return (it + 1, tmax, False, True, last_dm, False, tmean, lam)
        t_prev = tmean
    return (s["max_iters"], last_tmax, False, False, last_dm, False, last_tmean, lam)


@pytest.mark.parametrize("kw", [dict(max_iters=400, torque_threshold=2e-3),
                                dict(max_iters=400, torque_threshold=1e-9, dm_stop=3e-4, dm_samples=4,
                                     dm_min_iters=5),
                                dict(max_iters=300, torque_threshold=1e-9, dm_stop=None, min_iters_before_stall=5,
                                     stall_iters=4, stall_rel=0.2)])
def test_oracle_minimize_equals_python_restatement(orc, kw):
    g, mat, mask, m0, p = _setup(orc, 8, 6, "noise", 12)
    solver = orc.Solver(g, mat, mask)
    mo = m0.copy()
    ro = solver.minimize(mo, p, 2, orc.default_minimize_settings(**kw))
    mp = m0.copy()
    rp = _python_minimize(orc, solver, mp, p, 2, kw)
    got = (ro.iters, ro.final_torque, bool(ro.converged), bool(ro.stalled), ro.final_max_dm, bool(ro.dm_converged),
           ro.final_tmean, ro.final_lambda)
    assert got == rp
    assert np.array_equal(mo, mp)


# ------------------------------------------------------------------ relax_until_gate host logic

class _Rep:
    def __init__(self, ft, ftm=None, stop=E.STOP_TIGHTEN_FLOOR_REACHED):
        self.has_final_torque = 0 if ft is None else 1
        self.final_torque = 0.0 if ft is None else ft
        self.has_final_torque_max = 0 if ftm is None else 1
        self.final_torque_max = 0.0 if ftm is None else ftm
        self.stop_reason = stop


class _Scripted:
    """Replays canned relax reports and records the settings of every call."""

    def __init__(self, reps, tmax_now=1.0):
        self.reps = list(reps)
        self.calls = []
        self.tmax_now = tmax_now

    def relax(self, params, fmask, st):
        self.calls.append(("relax", E._copy(st)))
        return self.reps.pop(0)

    def minimize(self, params, fmask, st):
        self.calls.append(("minimize", st))
        return "mrep"

    def torque_metric(self, params, fmask, metric):
        assert metric == E.TORQUE_MAX
        self.calls.append(("tmax", None))
        return self.tmax_now


def test_relax_until_gate_first_pass_ok(orc):
    base = orc.default_relax_settings(has_final_torque_gate=1, final_torque_gate=1.0, gate_plateau_fails=3)
    s = _Scripted([_Rep(1e-4, 2e-3)])
    out = E.relax_until_gate(s, None, 2, base, E.RelaxGate(torque_gate=5e-4, torque_gate_max=5e-3))
    assert out.gate_passed and len(out.relax_passes) == 1 and not out.minimize_passes
    st = s.calls[0][1]
    # the inner gate is cleared, the rest is verbatim
    assert (st.has_final_torque_gate, st.has_final_torque_gate_max, st.gate_max_extra_accepted_steps,
            st.gate_plateau_fails) == (0, 0, 0, 0)
    assert st.max_err == base.max_err and st.phase1_enabled == base.phase1_enabled
    assert base.has_final_torque_gate == 1   # the caller's settings are untouched


def test_relax_until_gate_extra_passes_and_minimize(orc):
    base = orc.default_relax_settings(max_accepted_steps=1000, tighten_floor=1e-7)
    msett = orc.default_minimize_settings(max_iters=200, torque_threshold=8e-4)
    gate = E.RelaxGate(torque_gate=5e-4, extra_passes=3, fallback_to_minimize=True, minimize=msett,
                       extra_pass_max_steps_mult=2.5)
    # first pass fails, second fails, third passes; final_torque_max missing -> rebuilt
    s = _Scripted([_Rep(1e-3), _Rep(7e-4), _Rep(4e-4)], tmax_now=0.25)
    out = E.relax_until_gate(s, None, 2, base, gate)
    assert out.gate_passed
    assert len(out.relax_passes) == 3 and out.minimize_passes == ["mrep", "mrep"]
    kinds = [c[0] for c in s.calls]
    assert kinds == ["relax", "tmax", "minimize", "relax", "tmax", "minimize", "relax", "tmax"]
    for c in [c for c in s.calls if c[0] == "relax"][1:]:
        st = c[1]
        assert (st.phase1_enabled, st.phase2_enabled) == (0, 1)
        assert st.max_err == 1e-7
        assert st.has_torque_threshold == 0
        assert (st.torque_plateau_checks, st.torque_plateau_min_checks) == (1, 1)
        assert (st.torque_plateau_rel, st.torque_plateau_abs) == (0.0, 0.0)
        assert st.max_accepted_steps == 2500
    assert all(r.has_final_torque_max and r.final_torque_max == 0.25 for r in out.relax_passes)


def test_relax_until_gate_stops_on_max_accepted_steps(orc):
    base = orc.default_relax_settings()
    s = _Scripted([_Rep(1e-3), _Rep(1e-3, stop=E.STOP_MAX_ACCEPTED_STEPS), _Rep(1e-4)])
    out = E.relax_until_gate(s, None, 2, base, E.RelaxGate(torque_gate=5e-4, extra_passes=5))
    assert not out.gate_passed and len(out.relax_passes) == 2


def test_relax_until_gate_max_gate_and_missing_metric(orc):
    base = orc.default_relax_settings()
    # no final torque -> a metric gate fails (unwrap_or(inf)); the max gate reads final_torque_max
    s = _Scripted([_Rep(None, 1e-3), _Rep(1e-9, 1e-2), _Rep(1e-9, 1e-4)])
    out = E.relax_until_gate(s, None, 2, base, E.RelaxGate(torque_gate=1.0, torque_gate_max=1e-3, extra_passes=2))
    assert out.gate_passed and len(out.relax_passes) == 3
    assert not E.gate_ok(_Rep(None, 0.0), E.RelaxGate(torque_gate=1.0))
    assert E.gate_ok(_Rep(None, None), E.RelaxGate())


class _OracleSolver:
    """The oracle behind the solver-object interface that equilibrate.py drives."""

    def __init__(self, orc, solver, m):
        self.orc, self.s, self.m = orc, solver, m

    def relax(self, params, fmask, st):
        return self.s.relax(self.m, params, fmask, st)

    def minimize(self, params, fmask, st):
        return self.s.minimize(self.m, params, fmask, st)

    def torque_metric(self, params, fmask, metric):
        b = self.s.build_h_eff(self.m, tuple(params.b_ext), fmask)
        dp = C.POINTER(C.c_double)
        return self.orc.lib().orc_torque_metric(self.m.shape[0], self.m.ctypes.data_as(dp), b.ctypes.data_as(dp),
                                                metric)


def test_relax_until_gate_on_oracle(orc):
    g, mat, mask, m0, p = _setup(orc, 16, 12, "noise", 4)
    base = orc.default_relax_settings(torque_threshold=None, torque_metric=1, torque_plateau_checks=8,
                                      torque_plateau_min_checks=8, torque_plateau_rel=0.0, torque_plateau_abs=1e-7,
                                      max_err=1e-5, max_accepted_steps=400)
    gate = E.RelaxGate(torque_gate=1e-9, torque_gate_max=None, extra_passes=2, fallback_to_minimize=True,
                       minimize=orc.default_minimize_settings(max_iters=50, torque_threshold=8e-4))
    osv = _OracleSolver(orc, orc.Solver(g, mat, mask), m0.copy())
    out = E.relax_until_gate(osv, p, 2, base, gate)
    assert 1 <= len(out.relax_passes) <= 3
    assert len(out.minimize_passes) == len(out.relax_passes) - 1
    assert all(r.has_final_torque_max for r in out.relax_passes)
    assert out.gate_passed == E.gate_ok(out.relax_passes[-1], gate)
    assert np.allclose(np.linalg.norm(osv.m, axis=1), 1.0)


# ------------------------------------------------------------------ policies (equilibrate.rs:261-430)

def test_policy_defaults(gpu):
    """RemanencePolicy / HysteresisPolicy / RelaxGate defaults (equilibrate.rs:60-77, 270-300, 341-382)."""
    g = E.RelaxGate()
    assert (g.torque_gate, g.torque_gate_max, g.extra_passes, g.fallback_to_minimize,
            g.extra_pass_max_steps_mult) == (None, None, 2, False, 2.0)
    ms = g.minimize_settings()
    assert (ms.max_iters, ms.torque_threshold, ms.lambda0, ms.dm_stop) == (200, 8e-4, 2e-2, 1e-6)
    r = E.RemanencePolicy.default()
    assert r.reset_dt and r.gate.torque_gate == 5e-4 and r.gate.torque_gate_max is None
    st = r.relax
    assert (st.phase1_enabled, st.phase2_enabled, st.torque_metric, st.has_torque_threshold) == (1, 1, 1, 0)
    assert (st.torque_plateau_checks, st.torque_plateau_min_checks, st.torque_plateau_rel,
            st.torque_plateau_abs, st.max_err) == (8, 8, 0.0, 1e-7, 1e-5)
    h = E.HysteresisPolicy.default()
    assert h.premin is None and h.warm_start_dt and h.gate.torque_gate == 8e-4 and h.gate.torque_gate_max is None
    st = h.relax
    assert (st.phase1_enabled, st.phase2_enabled, st.torque_metric, st.has_torque_threshold) == (0, 1, 1, 0)
    assert (st.torque_plateau_checks, st.torque_plateau_min_checks, st.torque_plateau_rel,
            st.torque_plateau_abs) == (3, 5, 0.0, 0.0)


class _Params:
    def __init__(self, dt):
        self.dt = dt


def test_equilibrate_remanence_resets_dt(gpu):
    s = _Scripted([_Rep(1e-4, 1e-3)])
    p = _Params(3e-12)
    out = E.equilibrate_remanence(s, p, 2, E.RemanencePolicy.default())
    assert p.dt == 1e-13 and out.gate_passed and len(out.relax_passes) == 1


def test_hysteresis_step_dt_and_premin(gpu):
    """dt is reset on the first step or without warm start, kept otherwise; the optional
    minimiser pass runs before the gated relax (equilibrate.rs:395-430)."""
    pol = E.HysteresisPolicy.default()
    s = _Scripted([_Rep(1e-4), _Rep(1e-4)])
    p = _Params(3e-12)
    rep = E.hysteresis_step(s, p, 2, pol, is_first=False)
    assert p.dt == 3e-12 and rep.premin is None and rep.relax.gate_passed
    rep = E.hysteresis_step(s, p, 2, pol, is_first=True)
    assert p.dt == 1e-13
    pol.premin = gpu.MinimizeSettings.default(max_iters=10)
    pol.warm_start_dt = False
    s = _Scripted([_Rep(1e-4)])
    p = _Params(3e-12)
    rep = E.hysteresis_step(s, p, 2, pol, is_first=False)
    assert p.dt == 1e-13 and rep.premin == "mrep"
    assert [c[0] for c in s.calls][:2] == ["minimize", "relax"]
