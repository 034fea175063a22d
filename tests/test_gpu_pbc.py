"""Periodic-image demag on the GPU and the LLGDMAG v2 kernel cache, against the FP64 oracle."""
import struct

import numpy as np
import pytest

from helpers import case, gpu_solver

pytestmark = pytest.mark.gpu
MU0 = 4e-7 * np.pi


def _grids(gpu, orc, nx, ny, dx, dy, dz):
    return gpu.Grid2D(nx, ny, dx, dy, dz), orc.make_grid(nx, ny, dx, dy, dz)


@pytest.mark.parametrize("nx,ny,pbc", [(2, 128, (32, 0)), (3, 128, (32, 0)), (12, 10, (0, 3)), (16, 16, (2, 2)),
                                       (9, 7, (1, 0)), (20, 8, (0, 0))])
def test_pbc_field_matches_oracle(gpu, orc, nx, ny, pbc):
    gg, og = _grids(gpu, orc, nx, ny, 1e-9, 1e-9, 0.5e-9)
    m = orc.init_random(nx * ny, 17 + nx)
    op = gpu.DemagOp(gg, *pbc)
    b = op.field(8e5, m)
    bo = orc.demag_field_pbc(og, 8e5, pbc[0], pbc[1], m)
    assert np.abs(b - bo).max() <= 1e-10 * np.abs(bo).max()
    k = op.kspace()
    ko = orc.kernel_kspace_pbc(og, *pbc)
    assert np.abs(k - ko).max() <= 1e-11 * np.abs(ko).max()
    op.close()


def test_pbc_uniform_wire_averages(gpu, orc):
    """The reference's demag_2d_pbc driver: 2x128 cells repeated 32 times along x."""
    gg, og = _grids(gpu, orc, 2, 128, 1e-9, 1e-9, 0.5e-9)
    ms = 1.0 / MU0
    op = gpu.DemagOp(gg, 32, 0)
    for d in ((1, 0, 0), (0, 1, 0), (0, 0, 1)):
        m = np.tile(d, (256, 1)).astype(float)
        b = op.field(ms, m).mean(axis=0)
        bo = orc.demag_field_pbc(og, ms, 32, 0, m).mean(axis=0)
        assert np.allclose(b, bo, rtol=0, atol=1e-12)
    op.close()


def test_open_operator_equals_solver_demag(gpu, orc):
    c = case(24, 12)
    s = gpu_solver(gpu, c, gpu.FP64)
    m = orc.init_random(24 * 12, 8)
    s.set_state(m)
    b_s = s.compute_demag_field()
    op = gpu.DemagOp(gpu.Grid2D(24, 12, c["dx"], c["dy"], c["dz"]), 0, 0)
    b_o = op.field(c["ms"], m)
    assert np.abs(b_s - b_o).max() <= 1e-11 * np.abs(b_o).max()
    op.close()
    s.close()


def test_llgdmag_cache_round_trip(gpu, orc, tmp_path):
    nx, ny, pbc = 10, 6, (3, 0)
    gg, og = _grids(gpu, orc, nx, ny, 2e-9, 3e-9, 1e-9)
    ref_file = tmp_path / "oracle.bin"
    orc.write_llgdmag(og, *pbc, ref_file)
    # a file written by the oracle restatement of write_kernel_kspace is loaded as is
    op = gpu.DemagOp(gg, *pbc, cache_path=ref_file)
    assert op.loaded
    assert np.array_equal(op.kspace(), orc.kernel_kspace_pbc(og, *pbc))
    m = orc.init_random(nx * ny, 5)
    assert np.abs(op.field(7e5, m) - orc.demag_field_pbc(og, 7e5, *pbc, m)).max() < 1e-12 * 7e5
    op.close()
    # a missing file is built and written in the same layout
    mine = tmp_path / "sub" / "dir" / "gpu.bin"
    op = gpu.DemagOp(gg, *pbc, cache_path=mine)
    assert not op.loaded and mine.exists()
    a, b = ref_file.read_bytes(), mine.read_bytes()
    assert len(a) == len(b) and a[:68] == b[:68]
    da = np.frombuffer(a[68:], "<f8")
    db = np.frombuffer(b[68:], "<f8")
    assert np.abs(da - db).max() <= 1e-11 * np.abs(da).max()
    k_built = op.kspace()
    op.close()
    op = gpu.DemagOp(gg, *pbc, cache_path=mine)
    assert op.loaded and np.array_equal(op.kspace(), k_built)
    op.close()
    # a header that does not match (other cell size) is ignored and the kernel rebuilt
    g2 = gpu.Grid2D(nx, ny, 2e-9, 3e-9, 1.5e-9)
    op = gpu.DemagOp(g2, *pbc, cache_path=ref_file)
    assert not op.loaded
    op.close()
    assert struct.unpack("<7I", a[8:36]) == (2, nx, ny, 3, 0, nx, 2 * ny)
