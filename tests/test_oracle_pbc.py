"""Periodic-boundary demag and the LLGDMAG v2 cache file in the FP64 oracle.

Pins: the FFT field equals a direct circular convolution with the wrapped
kernel; pbc = (0, 0) through the periodic entry equals the open operator; a film
repeated many times in-plane with uniform mz sees B_z -> -mu0 Ms (thin-film
limit) and with uniform in-plane m a vanishing field; the file layout follows
write_kernel_kspace (demag_fft_uniform.rs:279-319)."""
import struct

import numpy as np
import pytest

MU0 = 4e-7 * np.pi


def _m(orc, n, seed):
    return orc.init_random(n, seed)


@pytest.mark.parametrize("nx,ny,pbc", [(6, 5, (2, 0)), (5, 7, (0, 3)), (4, 4, (1, 1)), (7, 3, (3, 2))])
def test_pbc_fft_equals_direct_circular_convolution(orc, nx, ny, pbc):
    g = orc.make_grid(nx, ny, 3e-9, 4e-9, 2e-9)
    m = _m(orc, nx * ny, 9 + nx)
    b = orc.demag_field_pbc(g, 8e5, pbc[0], pbc[1], m)
    d = orc.demag_field_direct_pbc(g, 8e5, pbc[0], pbc[1], m)
    assert np.abs(b - d).max() <= 1e-12 * np.abs(d).max()


def test_pbc_zero_equals_open_operator(orc):
    g = orc.make_grid(9, 6, 4e-9, 4e-9, 3e-9)
    mat = orc.make_material(8e5, 1.3e-11, 0.0, (0, 0, 1), None, True)
    m = _m(orc, 54, 3)
    b_open = orc.Solver(g, mat).demag_field(m)
    b_pbc = orc.demag_field_pbc(g, 8e5, 0, 0, m)
    assert np.array_equal(b_open, b_pbc)


def test_periodic_thin_film_limits(orc):
    nx = ny = 6
    g = orc.make_grid(nx, ny, 5e-9, 5e-9, 1e-9)
    ms = 1.0 / MU0
    mz = np.tile([0.0, 0.0, 1.0], (nx * ny, 1))
    bz = orc.demag_field_pbc(g, ms, 6, 6, mz).mean(axis=0)
    assert bz[2] == pytest.approx(-1.0, abs=2e-2)       # N_zz -> 1 for an infinite thin film
    assert abs(bz[0]) < 1e-12 and abs(bz[1]) < 1e-12
    mx = np.tile([1.0, 0.0, 0.0], (nx * ny, 1))
    bx = orc.demag_field_pbc(g, ms, 6, 6, mx).mean(axis=0)
    assert abs(bx[0]) < 2e-2                              # N_xx -> 0 in-plane


def test_llgdmag_file_layout(orc, tmp_path):
    g = orc.make_grid(6, 4, 2e-9, 3e-9, 1e-9)
    path = tmp_path / "k.bin"
    orc.write_llgdmag(g, 2, 0, path)
    raw = path.read_bytes()
    px, py = 6, 8
    assert len(raw) == 68 + 4 * px * py * 16
    assert raw[:8] == b"LLGDMAG\x00"
    assert struct.unpack("<7I", raw[8:36]) == (2, 6, 4, 2, 0, px, py)
    assert struct.unpack("<4d", raw[36:68]) == (2e-9, 3e-9, 1e-9, 10.0)
    data = np.frombuffer(raw[68:], dtype="<f8").view(np.complex128).reshape(4, py, px)
    assert np.array_equal(data, orc.kernel_kspace_pbc(g, 2, 0))
