"""The fused row pass (end of RK stage s + start of stage s+1 in one kernel) must
give exactly the bits of the unfused passes: same operations in the same order.
LLG_B200_NO_FUSE=1 selects the unfused kernels at solver creation; the column
form (staged or lean tables) is fixed by LLG_B200_COLUMN_FORM and must not change
the bits either."""
import numpy as np
import pytest

from helpers import GAMMA, case, gpu_solver, holes_mask, oracle_solver, random_m, rel_err

pytestmark = pytest.mark.gpu

CASES = [
    # nx, ny, dmi, ku, masked
    (1024, 64, 3e-3, 8e5, False),
    (256, 96, 1e-3, 0.0, True),
    (128, 34, None, 5e4, False),   # partial last row block
    (64, 64, -2e-3, 1e5, True),
]


def _pair(gpu, monkeypatch, c, prec, env):
    a = gpu_solver(gpu, c, prec)
    for k in env:
        monkeypatch.setenv(k, "1")
    b = gpu_solver(gpu, c, prec)
    for k in env:
        monkeypatch.delenv(k)
    return a, b


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("nx,ny,dmi,ku,masked", CASES)
def test_fused_rk45_equals_unfused(orc, gpu, monkeypatch, nx, ny, dmi, ku, masked, prec):
    msk = holes_mask(nx, ny, [(nx // 5, ny // 6, max(3, ny // 5))]) if masked else None
    c = case(nx, ny, dx=2e-9, dy=2e-9, dz=2e-9, ms=5.8e5, a_ex=1.5e-11, k_u=ku, dmi=dmi, mask=msk)
    fused, plain = _pair(gpu, monkeypatch, c, prec, ["LLG_B200_NO_FUSE"])
    m = random_m(orc, nx * ny, 31 + nx, msk)
    fused.set_state(m)
    plain.set_state(m)
    p1 = gpu.LLGParams(GAMMA, 0.3, 1e-14, (0.01, 0.0, 0.02))
    p2 = gpu.LLGParams(GAMMA, 0.3, 1e-14, (0.01, 0.0, 0.02))
    for _ in range(6):
        r1 = fused.step_rk45(p1, 2, 1e-5, 0.8, 1e-19, 1e-11)
        r2 = plain.step_rk45(p2, 2, 1e-5, 0.8, 1e-19, 1e-11)
        assert r1 == r2
        assert p1.dt == p2.dt
    a, r, _ = fused.run_rk45(p1, 2, 1e-5, 0.8, 1e-19, 1e-11, n_accepted=5)
    b, q, _ = plain.run_rk45(p2, 2, 1e-5, 0.8, 1e-19, 1e-11, n_accepted=5)
    assert (a, r) == (b, q)
    assert np.array_equal(fused.get_state(), plain.get_state())


@pytest.mark.parametrize("prec", [0, 1])
def test_fused_rk23_relax_equals_unfused(orc, gpu, monkeypatch, prec):
    nx, ny = 256, 64
    msk = holes_mask(nx, ny, [(20, 5, 9)])
    c = case(nx, ny, dmi=1e-3, mask=msk)
    fused, plain = _pair(gpu, monkeypatch, c, prec, ["LLG_B200_NO_FUSE"])
    m = random_m(orc, nx * ny, 4, msk)
    fused.set_state(m)
    plain.set_state(m)
    for s in (fused, plain):
        p = gpu.LLGParams(GAMMA, 0.5, 1e-13, (0.0, 0.01, 0.0))
        st = gpu.RelaxSettings.default(torque_threshold=1e-2, max_accepted_steps=300)
        s._rep = s.relax(p, 2, st)
    assert fused._rep.accepted_steps == plain._rep.accepted_steps
    assert np.array_equal(fused.get_state(), plain.get_state())


def test_fused_with_lean_column_equals_unfused_staged(orc, gpu, monkeypatch):
    """Fused rows + lean column (form 1) against unfused rows + staged column (form 0)."""
    nx, ny = 512, 1024
    c = case(nx, ny, dmi=2e-3)
    monkeypatch.setenv("LLG_B200_COLUMN_FORM", "1")
    lean = gpu_solver(gpu, c, 0)
    monkeypatch.setenv("LLG_B200_COLUMN_FORM", "0")
    monkeypatch.setenv("LLG_B200_NO_FUSE", "1")
    staged = gpu_solver(gpu, c, 0)
    monkeypatch.delenv("LLG_B200_COLUMN_FORM")
    monkeypatch.delenv("LLG_B200_NO_FUSE")
    assert lean.fft_plans()[1] == 1 and staged.fft_plans()[1] == 0
    m = random_m(orc, nx * ny, 77)
    lean.set_state(m)
    staged.set_state(m)
    assert np.array_equal(lean.compute_demag_field(), staged.compute_demag_field())
    p1 = gpu.LLGParams(GAMMA, 0.3, 1e-14, (0.01, 0.0, 0.02))
    p2 = gpu.LLGParams(GAMMA, 0.3, 1e-14, (0.01, 0.0, 0.02))
    a = lean.run_rk45(p1, 2, 1e-5, 0.8, 1e-19, 1e-11, n_accepted=4)
    b = staged.run_rk45(p2, 2, 1e-5, 0.8, 1e-19, 1e-11, n_accepted=4)
    assert a[:2] == b[:2]
    assert np.array_equal(lean.get_state(), staged.get_state())


@pytest.mark.parametrize("prec", [0, 1])
def test_odd_rows_with_power_of_two_width(orc, gpu, prec):
    """nx = 128 with an odd ny: FP32 takes the generic row kernels (the register-FFT
    row kernels need 16-byte aligned two-row pieces of the spectrum), FP64 the fast
    ones; both match the oracle."""
    nx, ny = 128, 33
    c = case(nx, ny, dmi=1e-3, k_u=5e4)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, prec)
    m = random_m(orc, nx * ny, 9)
    g.set_state(m)
    p = gpu.LLGParams(GAMMA, 0.1, 1e-13, (0.01, 0.0, 0.0))
    assert rel_err(g.build_h_eff(p, 2), o.build_h_eff(m, (0.01, 0.0, 0.0), 2)) <= (1e-9 if prec else 2e-5)
    po = orc.make_params(GAMMA, 0.1, 1e-13, (0.01, 0.0, 0.0))
    mo = m.copy()
    for _ in range(4):
        ro = o.step_rk45(mo, po, 2, 1e-5, 0.8, 1e-19, 1e-11)
        rg = g.step_rk45(p, 2, 1e-5, 0.8, 1e-19, 1e-11)
        assert ro[1] == rg[1]
        p.dt = po.dt
    assert np.abs(g.get_state() - mo).max() <= (1e-12 if prec else 1e-6)


def test_profile_reports_fused_pass(gpu):
    c = case(1024, 64)
    s = gpu_solver(gpu, c, 0)
    s.set_state(np.tile([1.0, 0.0, 0.0], (1024 * 64, 1)))
    ms = s.profile_stage(gpu.LLGParams(GAMMA, 0.02, 1e-13), 2, reps=3)
    assert ms.shape == (4,) and np.all(ms > 0)
