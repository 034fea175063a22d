"""Equilibration policies over the relax controller and the minimiser.

Host-side composition of the reference's equilibrate.rs: every relax pass and
every minimiser pass runs on the GPU (llg_relax / llg_minimize through the
solver object); this module only chooses the settings of the next pass and
reads the reports, as equilibrate.rs does on the CPU.

``solver`` is any object with the methods of ``llg_b200.Solver`` used here:
``relax(params, field_mask, settings)``, ``minimize(params, field_mask,
settings)`` and ``torque_metric(params, field_mask, metric)``.  Settings are
ctypes structures with the fields of RelaxSettings / MinimizeSettings.
"""
import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional

# RelaxStopReason order (relax.rs:39-45)
STOP_MAX_ACCEPTED_STEPS, STOP_PHASE2_DISABLED, STOP_TIGHTEN_FLOOR_REACHED, STOP_TORQUE_GATE_NOT_SATISFIED = 0, 1, 2, 3
TORQUE_MAX, TORQUE_MEAN = 0, 1


def _copy(st):
    c = type(st)()
    C.memmove(C.byref(c), C.byref(st), C.sizeof(st))
    return c


def _minimize_settings_gate_default(settings_cls):
    """MinimizeSettings::default() with max_iters 200 and threshold 8e-4 (equilibrate.rs:68-73)."""
    s = settings_cls.default()
    s.max_iters = 200
    s.torque_threshold = 8e-4
    return s


@dataclass
class RelaxGate:
    """RelaxGate (equilibrate.rs:34-77).  ``minimize`` None means the gate default
    (MinimizeSettings::default() with max_iters 200, torque_threshold 8e-4), built
    from ``minimize_settings_cls`` when a fallback pass needs it."""
    torque_gate: Optional[float] = None
    torque_gate_max: Optional[float] = None
    extra_passes: int = 2
    fallback_to_minimize: bool = False
    minimize: object = None
    extra_pass_max_steps_mult: float = 2.0
    minimize_settings_cls: object = None

    def minimize_settings(self):
        if self.minimize is not None:
            return self.minimize
        cls = self.minimize_settings_cls
        if cls is None:
            import llg_b200
            cls = llg_b200.MinimizeSettings
        return _minimize_settings_gate_default(cls)


@dataclass
class RelaxWithGateReport:
    """RelaxWithGateReport (equilibrate.rs:79-89)."""
    relax_passes: List[object] = field(default_factory=list)
    minimize_passes: List[object] = field(default_factory=list)
    gate_passed: bool = False


def _clear_inner_gate(s):
    # relax.rs's own gate is off: the policy owns gating (equilibrate.rs:175-179)
    s.has_final_torque_gate = 0
    s.has_final_torque_gate_max = 0
    s.final_torque_gate = 0.0
    s.final_torque_gate_max = 0.0
    s.gate_max_extra_accepted_steps = 0
    s.gate_plateau_fails = 0


def ensure_final_torque_max(solver, params, field_mask, rep):
    """equilibrate.rs:123-140: fill final_torque_max from a field rebuild when the
    relax pass left it unset (the value max |m x B| of the resident state)."""
    if not rep.has_final_torque_max:
        rep.final_torque_max = float(solver.torque_metric(params, field_mask, TORQUE_MAX))
        rep.has_final_torque_max = 1


def gate_ok(rep, gate):
    """equilibrate.rs:142-156."""
    ok_metric = True
    if gate.torque_gate is not None:
        ft = rep.final_torque if rep.has_final_torque else math.inf
        ok_metric = ft <= gate.torque_gate
    ok_max = True
    if gate.torque_gate_max is not None:
        fm = rep.final_torque_max if rep.has_final_torque_max else math.inf
        ok_max = fm <= gate.torque_gate_max
    return ok_metric and ok_max


def relax_until_gate(solver, params, field_mask, base_settings, gate):
    """relax_until_gate (equilibrate.rs:159-255): one relax pass with the caller's
    settings, then up to ``gate.extra_passes`` single-stage passes at the
    tighten floor with strict plateau semantics (optionally each preceded by a
    minimiser pass) until the torque gate passes."""
    out = RelaxWithGateReport()
    s0 = _copy(base_settings)
    _clear_inner_gate(s0)
    r0 = solver.relax(params, field_mask, s0)
    ensure_final_torque_max(solver, params, field_mask, r0)
    out.relax_passes.append(r0)
    if gate_ok(r0, gate):
        out.gate_passed = True
        return out
    for _ in range(int(gate.extra_passes)):
        if gate.fallback_to_minimize:
            out.minimize_passes.append(solver.minimize(params, field_mask, gate.minimize_settings()))
        s = _copy(base_settings)
        _clear_inner_gate(s)
        # single stage at the floor (equilibrate.rs:208-220)
        s.phase1_enabled = 0
        s.phase2_enabled = 1
        s.max_err = s.tighten_floor
        s.has_torque_threshold = 0
        s.torque_threshold = 0.0
        s.torque_plateau_checks = 1
        s.torque_plateau_min_checks = 1
        s.torque_plateau_rel = 0.0
        s.torque_plateau_abs = 0.0
        mult = max(float(gate.extra_pass_max_steps_mult), 1.0)
        s.max_accepted_steps = int(float(s.max_accepted_steps) * mult)
        r = solver.relax(params, field_mask, s)
        ensure_final_torque_max(solver, params, field_mask, r)
        out.relax_passes.append(r)
        if gate_ok(r, gate):
            out.gate_passed = True
            return out
        if r.stop_reason == STOP_MAX_ACCEPTED_STEPS:
            break
    out.gate_passed = gate_ok(out.relax_passes[-1], gate)
    return out


@dataclass
class RemanencePolicy:
    """RemanencePolicy (equilibrate.rs:261-300)."""
    relax: object
    gate: RelaxGate
    reset_dt: bool = True

    @classmethod
    def default(cls, relax_settings_cls=None):
        if relax_settings_cls is None:
            import llg_b200
            relax_settings_cls = llg_b200.RelaxSettings
        r = relax_settings_cls.default()
        r.phase1_enabled = 1
        r.phase2_enabled = 1
        r.torque_metric = TORQUE_MEAN
        r.has_torque_threshold = 0
        r.torque_threshold = 0.0
        r.torque_check_stride = 1
        r.torque_plateau_checks = 8
        r.torque_plateau_min_checks = 8
        r.torque_plateau_rel = 0.0
        r.torque_plateau_abs = 1e-7
        r.max_err = 1e-5
        g = RelaxGate(torque_gate=5e-4, torque_gate_max=None, extra_passes=2, fallback_to_minimize=False)
        return cls(relax=r, gate=g, reset_dt=True)


def equilibrate_remanence(solver, params, field_mask, policy):
    """equilibrate_remanence (equilibrate.rs:302-324)."""
    if policy.reset_dt:
        params.dt = 1e-13
    return relax_until_gate(solver, params, field_mask, policy.relax, policy.gate)


@dataclass
class HysteresisPolicy:
    """HysteresisPolicy (equilibrate.rs:326-382)."""
    relax: object
    gate: RelaxGate
    premin: object = None
    warm_start_dt: bool = True

    @classmethod
    def default(cls, relax_settings_cls=None):
        if relax_settings_cls is None:
            import llg_b200
            relax_settings_cls = llg_b200.RelaxSettings
        r = relax_settings_cls.default()
        r.phase1_enabled = 0
        r.phase2_enabled = 1
        r.torque_metric = TORQUE_MEAN
        r.has_torque_threshold = 0
        r.torque_threshold = 0.0
        r.torque_check_stride = 1
        r.torque_plateau_checks = 3
        r.torque_plateau_min_checks = 5
        r.torque_plateau_rel = 0.0
        r.torque_plateau_abs = 0.0
        r.max_err = 1e-5
        g = RelaxGate(torque_gate=8e-4, torque_gate_max=None, extra_passes=2, fallback_to_minimize=False)
        return cls(relax=r, gate=g, premin=None, warm_start_dt=True)


@dataclass
class HysteresisStepReport:
    """HysteresisStepReport (equilibrate.rs:384-388)."""
    premin: object
    relax: RelaxWithGateReport


def hysteresis_step(solver, params, field_mask, policy, is_first):
    """hysteresis_step (equilibrate.rs:395-430): optional minimiser pass, then the
    gated relax under the current params."""
    if not policy.warm_start_dt or is_first:
        params.dt = 1e-13
    premin = solver.minimize(params, field_mask, policy.premin) if policy.premin is not None else None
    return HysteresisStepReport(premin=premin,
                                relax=relax_until_gate(solver, params, field_mask, policy.relax, policy.gate))
