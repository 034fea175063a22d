"""CPU test of the SP4 driver's host logic (st_problems/sp4.rs:267-360) with a
scripted solver in place of the GPU film: the relax call and its settings, one
run call per 10 ps sample ending on the sample time, the table rows and their
number format, the OVF snapshot schedule and the <mx> = 0 crossover file."""
import math

import numpy as np
import pytest

from oracle import ovf as R


class _Report:
    accepted_steps = 1234


class _ScriptedFilm:
    def __init__(self, mx_of_k):
        self.mx_of_k = mx_of_k
        self.k = 0
        self.calls = []
        self.snapshots = []

    def set_state(self, m):
        self.calls.append(("set_state", m.shape, tuple(np.round(m[0], 12))))

    def torque_metric(self, params, fmask, metric):
        self.calls.append(("torque", metric))
        return 5e-5

    def relax(self, params, fmask, st):
        self.calls.append(("relax", params.dt, tuple(params.b_ext), fmask, st.has_torque_threshold,
                           st.torque_threshold, st.torque_plateau_checks, st.tighten_floor, st.max_accepted_steps))
        return _Report()

    def run_rk45(self, params, fmask, max_err, headroom, dt_min, dt_max, n_accepted=-1, t_end=math.inf,
                 max_attempts=-1):
        self.k += 1
        self.calls.append(("run", t_end, max_err, headroom, dt_min, dt_max, tuple(params.b_ext)))
        return 10, 1, t_end

    def mean_m(self):
        mx = self.mx_of_k(self.k)
        return np.array([mx, 0.1, 0.0])

    def write_ovf2(self, path, meta, fmt):
        self.snapshots.append((path.split("/")[-1], meta.desc_lines[-1], fmt))

    def close(self):
        self.calls.append(("close",))


def test_sp4_driver_schedule_and_outputs(gpu, tmp_path):
    import sp4

    film = _ScriptedFilm(lambda k: 0.9 - 0.07 * k)      # <mx> crosses zero at sample 13
    out = sp4.run_sp4("b", str(tmp_path / "sp4b"), t_total=2e-10, dt_out=1e-11, dt_ovf=1e-10, log=lambda *a: None,
                      solver=film)
    # start state, relax under zero field with the SP4 settings
    assert film.calls[0] == ("set_state", (10000, 3), tuple(np.round(np.array([1.0, 0.1, 0.0]) / math.sqrt(1.01), 12)))
    relax = [c for c in film.calls if c[0] == "relax"][0]
    assert relax == ("relax", 5e-14, (0.0, 0.0, 0.0), gpu.FULL, 1, 1e-4, 0, 1e-9, 2000000)
    # one run call per sample, each ending on the sample time, under field b
    runs = [c for c in film.calls if c[0] == "run"]
    assert len(runs) == 20
    for k, c in enumerate(runs, start=1):
        assert c[1] == pytest.approx(1e-11, rel=1e-12)
        assert c[2:6] == (1e-5, 0.8, 1e-13 * 1e-6, 1e-13 * 100.0)   # dt0_run * 1e-6 / * 100 (sp4.rs:166-167)
        assert c[6] == (-35.5e-3, -6.3e-3, 0.0)
    assert film.calls[-1] == ("close",)
    # table: header, t = 0 row, then one row per sample in Rust's {:.16e}
    lines = (tmp_path / "sp4b" / "table.csv").read_text().splitlines()
    assert lines[0] == "t_s,mx,my,mz" and len(lines) == 22
    for k, line in enumerate(lines[1:]):
        t, mx, my, mz = line.split(",")
        assert t == R.rust_exp(k * 1e-11, 16)
        assert mx == R.rust_exp(0.9 - 0.07 * k, 16) and my == R.rust_exp(0.1, 16) and mz == R.rust_exp(0.0, 16)
    # snapshots: t = 0, every 100 ps, and the crossover file at the first <mx> <= 0 sample
    names = [s[0] for s in film.snapshots]
    assert names == ["m0000000.ovf", "m0000001.ovf", "m_mx_zero.ovf", "m0000002.ovf"]
    assert all(s[2] == gpu.OVF_TEXT for s in film.snapshots)
    times = {s[0]: s[1] for s in film.snapshots}
    assert times["m_mx_zero.ovf"] == f"Total simulation time:  {R.rust_exp(13 * 1e-11, 16)}  s"
    assert times["m0000002.ovf"] == f"Total simulation time:  {R.rust_exp(20 * 1e-11, 16)}  s"
    assert out["crossover_t"] == 13 * 1e-11 and out["snapshots"] == 3
    assert out["run_accepted"] == 200 and out["run_rejected"] == 20 and out["relax_accepted"] == 1234


def test_sp4_no_crossover_and_case_fallback(gpu, tmp_path):
    import sp4

    film = _ScriptedFilm(lambda k: 0.5)
    out = sp4.run_sp4("x", str(tmp_path / "o"), t_total=5e-11, dt_out=1e-11, dt_ovf=1e-10, log=lambda *a: None,
                      solver=film)
    assert out["crossover_t"] is None
    assert [s[0] for s in film.snapshots] == ["m0000000.ovf"]
    assert [c for c in film.calls if c[0] == "run"][0][6] == (-24.6e-3, 4.3e-3, 0.0)   # an unknown case is 'a'
