"""CPU test of the device relax controller's logic.

The GPU runs relax_with_report (relax.rs:334-768) as a per-film state machine
(relax_control_core in relax_dev.cuh).  Here the same source is compiled for
the host and driven by the FP64 oracle's energy / torque / RK23 primitives;
with identical arithmetic underneath, every report field and the final state
must equal the oracle's own restatement of relax_with_report."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from helpers import GAMMA, case, holes_mask

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
FIELDS = ["accepted_steps", "rejected_steps", "torque_checks", "torque_field_rebuilds", "stop_reason",
          "last_stage_stop", "has_final_torque", "final_torque", "has_final_torque_max", "final_torque_max",
          "final_max_err", "final_dt"]


@pytest.fixture(scope="module")
def harness(orc, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("harness") / "libharness.so")
    odir = os.path.join(ROOT, "oracle")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-I/usr/local/cuda/include",
                    os.path.join(HERE, "harness", "relax_sm_harness.cpp"), "-o", out, "-L", odir, "-loracle",
                    "-Wl,-rpath," + odir], check=True)
    H = C.CDLL(out)
    dp = C.POINTER(C.c_double)
    H.harness_relax.argtypes = [C.POINTER(orc.Grid), C.POINTER(orc.Material), C.c_void_p, dp, C.POINTER(orc.Params),
                                C.c_int, C.POINTER(orc.RelaxSettings), C.POINTER(orc.RelaxReport), C.c_longlong]
    return H


SCENARIOS = [
    ("threshold", dict(torque_threshold=1e-3, max_accepted_steps=20000), (0.05, 0, 0), None),
    ("plateau_f32_phase1_cap", dict(torque_threshold=None, torque_metric=3, torque_plateau_checks=1,
                                    torque_plateau_min_checks=1, torque_plateau_rel=0.0, torque_plateau_abs=0.0,
                                    rel_energy_tol=0.0, max_accepted_steps=3000), (0, 0, 0.01), None),
    ("plateau_energy_tol", dict(torque_threshold=None, torque_metric=3, torque_plateau_checks=1,
                                torque_plateau_min_checks=1, torque_plateau_rel=0.0, torque_plateau_abs=0.0,
                                rel_energy_tol=1e-9, max_accepted_steps=3000), (0, 0, 0.01), None),
    ("plateau_mean_no_phase1", dict(torque_threshold=None, torque_metric=1, torque_plateau_checks=3,
                                    torque_plateau_min_checks=2, max_accepted_steps=5000, phase1_enabled=0),
     (0.05, 0, 0), None),
    ("gate", dict(torque_threshold=1e-3, has_final_torque_gate_max=1, final_torque_gate_max=1e-5,
                  gate_max_extra_accepted_steps=500, gate_plateau_fails=3, max_accepted_steps=20000), (0.05, 0, 0),
     None),
    ("masked_dmi", dict(torque_threshold=1e-3, max_accepted_steps=20000), (0.01, 0, 0), "holes"),
]


@pytest.mark.parametrize("name,kw,bext,maskkind", SCENARIOS, ids=[s[0] for s in SCENARIOS])
def test_device_relax_controller_equals_relax_with_report(orc, harness, name, kw, bext, maskkind):
    if maskkind == "holes":
        mask = holes_mask(32, 32, [(4, 2, 6)])
        c = case(32, 32, dmi=1e-3, mask=mask)
        m0 = orc.init_random(1024, 70)
        m0[mask == 0] = 0.0
    else:
        mask = None
        c = case(16, 12)
        m0 = orc.init_random(16 * 12, 4)
    g = orc.make_grid(c["nx"], c["ny"], c["dx"], c["dy"], c["dz"])
    mat = orc.make_material(c["ms"], c["a_ex"], c["k_u"], c["easy"], c["dmi"], c["demag"])
    mo = m0.copy()
    po = orc.make_params(GAMMA, 0.5, 1e-13, bext)
    ro = orc.Solver(g, mat, mask).relax(mo, po, 2, orc.default_relax_settings(**kw))
    mh = m0.copy()
    ph = orc.make_params(GAMMA, 0.5, 1e-13, bext)
    rh = orc.RelaxReport()
    mp = None
    if mask is not None:
        mk = np.ascontiguousarray(mask.astype(np.uint8))
        mp = mk.ctypes.data_as(C.c_void_p)
    rc = harness.harness_relax(C.byref(g), C.byref(mat), mp, mh.ctypes.data_as(C.POINTER(C.c_double)), C.byref(ph), 2,
                               C.byref(orc.default_relax_settings(**kw)), C.byref(rh), 10 ** 7)
    assert rc == 0
    for f in FIELDS:
        assert getattr(rh, f) == getattr(ro, f), f
    assert np.array_equal(mh, mo)
