"""OVF 2.0 files of a solver's resident state (binary4 packed to f32 on the
GPU): byte-identical to the restated writers applied to the state read back."""
import numpy as np
import pytest

from helpers import case, gpu_solver
from oracle import ovf as R

pytestmark = pytest.mark.gpu
LABELS, UNITS = ("m_x", "m_y", "m_z"), ("1", "1", "1")


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("fmt", ["binary4", "text"])
def test_state_writer_bytes(orc, gpu, tmp_path, prec, fmt):
    nx, ny = 96, 40
    c = case(nx, ny)
    s = gpu_solver(gpu, c, prec)
    s.set_state(orc.init_random(nx * ny, 17))
    meta = gpu.OvfMeta.magnetization().with_total_sim_time(2.5e-11)
    p = tmp_path / f"state.{fmt}.ovf"
    s.write_ovf2(p, meta, gpu.OVF_BINARY4 if fmt == "binary4" else gpu.OVF_TEXT)
    m = s.get_state()
    make = R.ovf2_binary4_bytes if fmt == "binary4" else R.ovf2_text_bytes
    assert p.read_bytes() == make(nx, ny, c["dx"], c["dy"], c["dz"], m, "m", meta.desc_lines, LABELS, UNITS)


def test_batch_film_writer(orc, gpu, tmp_path):
    grids = [gpu.Grid2D(32, 16, 4e-9, 4e-9, 3e-9), gpu.Grid2D(24, 24, 3e-9, 3e-9, 3e-9)]
    mats = [gpu.Material(8e5, 1.3e-11, demag=True)] * 2
    b = gpu.Batch(grids, mats, gpu.FP32)
    for f, g in enumerate(grids):
        b.set_state(f, orc.init_random(g.nx * g.ny, 40 + f))
    for f, g in enumerate(grids):
        p = tmp_path / f"film{f}.ovf"
        b.write_ovf2(f, p, gpu.OvfMeta.magnetization())
        m = b.get_state(f)
        assert p.read_bytes() == R.ovf2_binary4_bytes(g.nx, g.ny, g.dx, g.dy, g.dz, m, "m", [], LABELS, UNITS)
    with pytest.raises(gpu.LLGError):
        b.write_ovf2(2, tmp_path / "x.ovf", gpu.OvfMeta.magnetization())
