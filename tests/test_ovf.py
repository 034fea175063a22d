"""OVF 2.0 writers (ovf.rs:17-316): the library's files are byte-identical to a
pure-Python restatement of write_ovf2_rectangular_text / _binary4, whose number
format (Rust's `{:.<p>e}`) is computed with exact decimal arithmetic.  Host
arrays only: no GPU is used here."""
import math
import struct

import numpy as np
import pytest

from oracle import ovf as R

LABELS, UNITS = ("m_x", "m_y", "m_z"), ("1", "1", "1")


def _special_values():
    return [0.0, -0.0, 1.0, -1.0, 0.5, 2.0 ** -17, -(2.0 ** -17), 3 * 2.0 ** -20, 1e-300, 5e-324, 1.7976931348623157e308,
            9.99999999995, 0.1, 1.0 / 3.0, 123456.789, -7.62939453125e-6]


def test_rust_exp_matches_exact_decimal_restatement(gpu):
    rng = np.random.default_rng(5)
    vals = _special_values() + list(rng.standard_normal(300)) + list(10.0 ** rng.uniform(-30, 30, 300))
    # dyadic values whose 11th or 18th significant digit is an exact tie
    vals += [k * 2.0 ** -e for k in (1, 3, 5, 7, 9, 11) for e in range(14, 40)]
    for v in vals:
        for p in (3, 10, 16, 17):
            assert gpu.rust_exp(v, p) == R.rust_exp(v, p), (v, p)
    assert gpu.rust_exp(float("nan"), 10) == "NaN" and gpu.rust_exp(-math.inf, 3) == "-inf"
    # ties to even: 2^-17 = 7.62939453125e-6
    assert R.rust_exp(2.0 ** -17, 10) == "7.6293945312e-6"
    assert R.rust_exp(1.0, 10) == "1.0000000000e0" and R.rust_exp(123456.0, 3) == "1.235e5"


def _field(nx, ny, seed):
    rng = np.random.default_rng(seed)
    m = rng.standard_normal((nx * ny, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    sp = _special_values()[:12]
    m[: len(sp), 0] = sp
    return m


@pytest.mark.parametrize("fmt", ["text", "binary4"])
def test_host_writer_bytes_equal_restatement(gpu, tmp_path, fmt):
    nx, ny, dx, dy, dz = 7, 5, 4e-9, 3.5e-9, 1e-9
    m = _field(nx, ny, 1)
    meta = gpu.OvfMeta.magnetization().with_total_sim_time(1.2345e-10)
    meta.push_desc_line("stage 3 of 7")
    path = tmp_path / "deep" / "dir" / f"m.{fmt}.ovf"      # parent directories are created
    g = gpu.Grid2D(nx, ny, dx, dy, dz)
    if fmt == "text":
        gpu.write_ovf2_rectangular_text(path, g, m, meta)
        want = R.ovf2_text_bytes(nx, ny, dx, dy, dz, m, "m", meta.desc_lines, LABELS, UNITS)
    else:
        gpu.write_ovf2_rectangular_binary4(path, g, m, meta)
        want = R.ovf2_binary4_bytes(nx, ny, dx, dy, dz, m, "m", meta.desc_lines, LABELS, UNITS)
    got = path.read_bytes()
    assert got == want
    assert meta.desc_lines[0] == "Total simulation time:  1.2345000000000000e-10  s"


def test_binary4_layout(gpu, tmp_path):
    nx, ny = 3, 2
    m = np.arange(18, dtype=np.float64).reshape(6, 3) * 0.25
    p = tmp_path / "b.ovf"
    gpu.write_ovf2_rectangular_binary4(p, gpu.Grid2D(nx, ny, 1e-9, 1e-9, 1e-9), m, gpu.OvfMeta.magnetization())
    raw = p.read_bytes()
    start = raw.index(b"# Begin: Data Binary 4\n") + len(b"# Begin: Data Binary 4\n")
    assert struct.unpack("<f", raw[start:start + 4])[0] == 1234567.0
    vals = np.frombuffer(raw[start + 4:start + 4 + 72], dtype="<f4").reshape(6, 3)
    assert np.array_equal(vals, m.astype(np.float32))
    assert raw[start + 76:] == b"\n# End: Data Binary 4\n# End: Segment\n# End: File\n"


def test_larger_text_file_parallel_formatting(gpu, tmp_path):
    """More cells than one formatting chunk: the chunks are written in order."""
    nx, ny = 200, 180
    m = _field(nx, ny, 2)
    p = tmp_path / "big.ovf"
    gpu.write_ovf2_rectangular_text(p, gpu.Grid2D(nx, ny, 2e-9, 2e-9, 2e-9), m, gpu.OvfMeta.magnetization())
    assert p.read_bytes() == R.ovf2_text_bytes(nx, ny, 2e-9, 2e-9, 2e-9, m, "m", [], LABELS, UNITS)


def test_errors_are_statuses(gpu, tmp_path):
    blocker = tmp_path / "file"
    blocker.write_text("x")
    with pytest.raises(gpu.LLGError):
        gpu.write_ovf2_rectangular_binary4(blocker / "sub" / "m.ovf", gpu.Grid2D(2, 2, 1e-9, 1e-9, 1e-9),
                                           np.zeros((4, 3)), gpu.OvfMeta.magnetization())


def test_ovf_series_schedule(gpu, tmp_path):
    """OvfSeries (ovf.rs:255-316): frame 0 at t = 0, then one frame per `every` the
    simulated time has passed (several at once after a long step)."""
    written = []
    s = gpu.OvfSeries(str(tmp_path / "series"), 1e-11)
    mk = lambda k, t: f"f{k:05d}_{t:.3e}"
    s.dump_initial(lambda path, meta: written.append(path), mk, gpu.OvfMeta.magnetization())
    for t in (0.4e-11, 1.0e-11, 1.2e-11, 3.5e-11, 3.6e-11):
        s.maybe_dump_due(lambda path, meta: written.append(path), t, mk,
                         lambda tt: gpu.OvfMeta.magnetization().with_total_sim_time(tt))
    assert written == [mk(0, 0.0), mk(1, 1e-11), mk(2, 2e-11), mk(3, 3e-11)]
    assert s.frame == 4 and s.next_dump == pytest.approx(4e-11)
    off = gpu.OvfSeries(str(tmp_path / "off"), 0.0)
    off.maybe_dump_due(lambda path, meta: written.append(path), 1.0, mk, None)
    assert len(written) == 4
