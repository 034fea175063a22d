"""The SP4 driver flow (st_problems/sp4.rs) on the GPU, shortened to 100 ps:
table.csv and the text OVF snapshots in the reference's formats."""
import numpy as np
import pytest

from oracle import ovf as R

pytestmark = pytest.mark.gpu


def test_sp4_short_run_outputs(gpu, tmp_path):
    import sp4

    out = sp4.run_sp4("a", str(tmp_path / "sp4a"), precision=gpu.FP32, t_total=1e-10, dt_out=1e-11, dt_ovf=5e-11,
                      log=lambda *a: None)
    assert out["relax_torque"] <= 1e-4 * 1.02      # FP32 field allowance on the SP4 threshold
    lines = (tmp_path / "sp4a" / "table.csv").read_text().splitlines()
    assert lines[0] == "t_s,mx,my,mz" and len(lines) == 12
    for k, line in enumerate(lines[1:]):
        f = line.split(",")
        assert len(f) == 4
        assert f[0] == R.rust_exp(k * 1e-11, 16)
        assert all(x == R.rust_exp(float(x), 16) for x in f)
    names = sorted(p.name for p in (tmp_path / "sp4a").glob("m*.ovf"))
    assert names == ["m0000000.ovf", "m0000001.ovf", "m0000002.ovf"]
    # the last snapshot is the final state: its mean equals the table's last row
    text = (tmp_path / "sp4a" / "m0000002.ovf").read_text().splitlines()
    assert text[0] == "# OOMMF OVF 2.0"
    # the snapshot time is k * dt_out as sp4.rs:309 computes it
    assert "# Desc: Total simulation time:  " + R.rust_exp(10 * 1e-11, 16) + "  s" in text
    i0 = text.index("# Begin: Data Text") + 1
    data = np.array([[float(x) for x in ln.split()] for ln in text[i0:i0 + 200 * 50]])
    assert np.abs(np.linalg.norm(data, axis=1) - 1.0).max() < 1e-6
    last = [float(x) for x in lines[-1].split(",")[1:]]
    assert np.abs(data.mean(axis=0) - last).max() < 1e-9
    # under field a the film starts to switch: <mx> falls from its relaxed value
    first = [float(x) for x in lines[1].split(",")[1:]]
    assert last[0] < first[0]
