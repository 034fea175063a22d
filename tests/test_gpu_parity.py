"""GPU (sm_100a) vs CPU FP64 oracle parity, through the C ABI.

Tolerances (relative to the largest reference magnitude):
  FP64 path: 1e-9 for fields and kernels (FFT round-off plus FMA contraction),
  FP32 path: 2e-5 for fields (single-precision FFT of 2L points).
"""
import numpy as np
import pytest

from helpers import GAMMA, case, gpu_solver, holes_mask, oracle_solver, random_m, rel_err

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (2, 2), (3, 5), (1, 7), (7, 1), (12, 10), (11, 13), (64, 32), (96, 64), (128, 32)]
TOL = {0: 2e-5, 1: 1e-9}


@pytest.mark.parametrize("nx,ny", SHAPES)
def test_kernel_spectrum_matches_oracle(orc, gpu, nx, ny):
    c = case(nx, ny)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, gpu.FP64)
    ko = o.kernel_kspace()  # [4, py, px] complex
    kg = g.kernel_kspace()  # [4, ny+1, nx+1]
    ref = ko[:, : ny + 1, : nx + 1].real
    for comp in range(4):
        scale = np.abs(ko[comp].real).max()
        assert np.abs(kg[comp] - ref[comp]).max() <= 1e-11 * max(scale, 1e-300), comp


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("nx,ny", SHAPES)
def test_demag_field_matches_oracle(orc, gpu, nx, ny, prec):
    c = case(nx, ny)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, prec)
    m = random_m(orc, nx * ny, 1234 + nx)
    g.set_state(m)
    bo = o.demag_field(m)
    bg = g.compute_demag_field()
    assert rel_err(bg, bo) <= TOL[prec]


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("fmask", [0, 1, 2])
@pytest.mark.parametrize("nx,ny,dmi,ku", [(16, 12, 3e-3, 8e5), (33, 20, None, 5e2), (1, 9, 1e-4, 0.0), (64, 64, -2e-3, 1e5)])
def test_effective_field_matches_oracle(orc, gpu, nx, ny, dmi, ku, fmask, prec):
    c = case(nx, ny, dx=2e-9, dy=2e-9, dz=2e-9, ms=5.8e5, a_ex=1.5e-11, k_u=ku, easy=(0.2, -0.3, 0.93), dmi=dmi)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, prec)
    m = random_m(orc, nx * ny, 99)
    g.set_state(m)
    bext = (0.01, -0.02, 0.005)
    p = gpu.LLGParams(GAMMA, 0.3, 1e-13, bext)
    bo = o.build_h_eff(m, bext, fmask)
    bg = g.build_h_eff(p, fmask)
    assert rel_err(bg, bo) <= TOL[prec]


@pytest.mark.parametrize("prec", [0, 1])
def test_masked_field_and_energy(orc, gpu, prec):
    nx, ny = 48, 40
    msk = holes_mask(nx, ny, [(5, 3, 6), (-12, -8, 4)])
    c = case(nx, ny, dmi=1.5e-3, mask=msk)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, prec)
    m = random_m(orc, nx * ny, 7, msk)
    g.set_state(m)
    bext = (0.02, 0.0, 0.0)
    p = gpu.LLGParams(GAMMA, 0.5, 1e-13, bext)
    assert rel_err(g.build_h_eff(p, 2), o.build_h_eff(m, bext, 2)) <= TOL[prec]
    eo, eg = o.energy(m, bext), g.compute_energy(bext)
    for term in ("exchange", "anisotropy", "zeeman", "dmi", "demag"):
        ref = getattr(eo, term)
        assert abs(getattr(eg, term) - ref) <= (1e-10 if prec else 2e-5) * max(abs(eo.total()), 1e-300), term


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("nx,ny,dmi,ku", [(32, 24, None, 0.0), (20, 20, 3e-3, 8e5), (5, 3, 1e-3, 1e5)])
def test_energy_matches_oracle(orc, gpu, nx, ny, dmi, ku, prec):
    c = case(nx, ny, k_u=ku, dmi=dmi)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, prec)
    m = random_m(orc, nx * ny, 5)
    g.set_state(m)
    bext = (0.01, 0.02, -0.03)
    eo, eg = o.energy(m, bext), g.compute_energy(bext)
    for term in ("exchange", "anisotropy", "zeeman", "dmi", "demag"):
        ref = getattr(eo, term)
        tol = (1e-10 if prec else 2e-5) * max(abs(ref), abs(eo.total()) * 1e-3, 1e-300)
        assert abs(getattr(eg, term) - ref) <= tol, term


@pytest.mark.parametrize("prec", [0, 1])
def test_rk45_steps_match_oracle(orc, gpu, prec):
    nx, ny = 24, 16
    c = case(nx, ny, dmi=1e-3, k_u=2e4)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, prec)
    m = orc.init_uniform_with_noise(nx * ny, (1, 0, 0), 0.2, 42)
    g.set_state(m)
    po = orc.make_params(GAMMA, 0.02, 1e-13, (0.01, 0.015, 0.0))
    pg = gpu.LLGParams(GAMMA, 0.02, 1e-13, (0.01, 0.015, 0.0))
    mo = m.copy()
    args = (2, 1e-5, 0.8, 1e-19, 1e-11)
    for step in range(12):
        ro = o.step_rk45(mo, po, *args)
        rg = g.step_rk45(pg, *args)
        assert ro[1] == rg[1], step
        assert rg[2] == pytest.approx(ro[2], rel=1e-12 if prec else 1e-5)
        # measured worst case over the 12 steps: 5.8e-11 (FP64), 2.8e-3 (FP32)
        assert rg[0] == pytest.approx(ro[0], rel=1e-9 if prec else 1e-2), step
        pg.dt = po.dt  # keep the step sequences identical (replayed dt)
    mg = g.get_state()
    assert np.abs(mg - mo).max() <= (1e-12 if prec else 1e-6)   # measured 1.6e-14 / 1.2e-7


@pytest.mark.parametrize("prec", [0, 1])
def test_rk23_relax_steps_match_oracle(orc, gpu, prec):
    nx, ny = 20, 12
    c = case(nx, ny, dmi=1e-3)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, prec)
    m = orc.init_random(nx * ny, 3)
    g.set_state(m)
    po = orc.make_params(GAMMA, 0.5, 1e-13, (0.0, 0.0, 0.01))
    pg = gpu.LLGParams(GAMMA, 0.5, 1e-13, (0.0, 0.0, 0.01))
    mo = m.copy()
    args = (2, 1e-5, 0.8, 1e-18, 1e-11)
    for step in range(10):
        ro = o.step_rk23_relax(mo, po, *args)
        rg = g.step_rk23_relax(pg, *args)
        assert ro[1] == rg[1], step
        # measured worst case over the 10 steps: 5.2e-11 (FP64), 5.6e-4 (FP32)
        assert rg[0] == pytest.approx(ro[0], rel=1e-9 if prec else 3e-3), step
        pg.dt = po.dt
    assert np.abs(g.get_state() - mo).max() <= (1e-12 if prec else 1e-6)   # measured 9.0e-15 / 2.1e-7


@pytest.mark.parametrize("prec", [0, 1])
def test_torque_metrics_match_oracle(orc, gpu, prec):
    nx, ny = 30, 18
    c = case(nx, ny, dmi=2e-3)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, prec)
    m = random_m(orc, nx * ny, 11)
    g.set_state(m)
    bext = (0.0, 0.01, 0.0)
    b = o.build_h_eff(m, bext, 2)
    p = gpu.LLGParams(GAMMA, 0.5, 1e-13, bext)
    for metric in range(4):
        ref = orc.torque_metric(m, b, metric)
        assert g.torque_metric(p, 2, metric) == pytest.approx(ref, rel=1e-10 if prec else 1e-5)


def test_run_rk45_device_loop_matches_single_steps(gpu, orc):
    nx, ny = 32, 16
    c = case(nx, ny)
    m = orc.init_uniform_with_noise(nx * ny, (1, 0, 0), 0.1, 5)
    g1 = gpu_solver(gpu, c, gpu.FP64)
    g2 = gpu_solver(gpu, c, gpu.FP64)
    g1.set_state(m)
    g2.set_state(m)
    p1 = gpu.LLGParams(GAMMA, 0.02, 1e-13, (0.02, 0.0, 0.0))
    p2 = gpu.LLGParams(GAMMA, 0.02, 1e-13, (0.02, 0.0, 0.0))
    acc = 0
    while acc < 25:
        _, a, _ = g1.step_rk45(p1, 2, 1e-6, 0.8, 1e-19, 1e-11)
        acc += a
    a, r, t = g2.run_rk45(p2, 2, 1e-6, 0.8, 1e-19, 1e-11, n_accepted=25)
    assert a == 25
    assert np.array_equal(g1.get_state(), g2.get_state())
    assert p1.dt == p2.dt


def test_mean_m_and_state_roundtrip(gpu, orc):
    c = case(40, 30)
    g = gpu_solver(gpu, c, gpu.FP64)
    m = orc.init_random(1200, 8)
    g.set_state(m)
    assert np.array_equal(g.get_state(), m)
    assert np.allclose(g.mean_m(), m.mean(axis=0), atol=1e-14)


FAST_SHAPES = [(16, 16), (32, 64), (64, 128), (128, 256), (256, 32), (512, 16), (1024, 64), (2048, 16), (16, 2048),
               (64, 1024)]


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("nx,ny", FAST_SHAPES)
def test_register_fft_path_matches_oracle(orc, gpu, nx, ny, prec):
    """Power-of-two sizes run the register-FFT kernels; fields must match the oracle."""
    if prec == 1 and max(nx, ny) > 1024:
        pytest.skip("FP64 in-shared-memory transforms are limited to 1024")
    c = case(nx, ny, dmi=2e-3, k_u=1e5)
    o = oracle_solver(orc, c)
    g = gpu_solver(gpu, c, prec)
    m = random_m(orc, nx * ny, 21 + nx + ny)
    g.set_state(m)
    bext = (0.01, 0.0, -0.02)
    p = gpu.LLGParams(GAMMA, 0.1, 1e-13, bext)
    assert rel_err(g.build_h_eff(p, 2), o.build_h_eff(m, bext, 2)) <= TOL[prec]
    assert rel_err(g.compute_demag_field(), o.demag_field(m)) <= TOL[prec]


@pytest.mark.parametrize("nx,ny", [(256, 256), (128, 64), (1024, 32)])
def test_register_fft_matches_generic_kernels(orc, gpu, nx, ny, monkeypatch):
    c = case(nx, ny)
    m = random_m(orc, nx * ny, 5)
    fast = gpu_solver(gpu, c, gpu.FP64)
    monkeypatch.setenv("LLG_B200_GENERIC_FFT", "1")
    gen = gpu_solver(gpu, c, gpu.FP64)
    monkeypatch.delenv("LLG_B200_GENERIC_FFT")
    fast.set_state(m)
    gen.set_state(m)
    p = gpu.LLGParams(GAMMA, 0.02, 1e-13, (0.0, 0.01, 0.0))
    assert rel_err(fast.build_h_eff(p, 2), gen.build_h_eff(p, 2)) <= 1e-12
    for _ in range(3):
        rf = fast.step_rk45(p, 2, 1e-5, 0.8, 1e-19, 1e-11)
        p.dt = rf[2]
        rg = gen.step_rk45(p, 2, 1e-5, 0.8, 1e-19, 1e-11)
        assert rf[1] == rg[1]
        p.dt = rf[2]
    assert np.abs(fast.get_state() - gen.get_state()).max() <= 1e-12


PLAN1_SHAPES = [(1024, 128, 0), (2048, 256, 0), (64, 1024, 0), (512, 256, 1), (128, 512, 1)]


@pytest.mark.parametrize("nx,ny,prec", [(256, 1024, 0), (128, 256, 1)])
def test_column_forms_give_the_same_bits(orc, gpu, monkeypatch, nx, ny, prec):
    """Every column form (plan 0/1, staged / lean, fixed by LLG_B200_COLUMN_FORM) gives
    the same field as the other form of the same plan: the lean form only reads its
    tables from another memory."""
    m = random_m(orc, nx * ny, 3 + ny)
    c = case(nx, ny, dmi=1e-3)
    out = {}
    for form in range(4):
        monkeypatch.setenv("LLG_B200_COLUMN_FORM", str(form))
        s = gpu_solver(gpu, c, prec)
        monkeypatch.delenv("LLG_B200_COLUMN_FORM")
        assert s.fft_plans()[1] == form
        s.set_state(m)
        out[form] = s.compute_demag_field()
        s.close()
    assert np.array_equal(out[0], out[1])
    assert np.array_equal(out[2], out[3])
    assert rel_err(out[0], out[2]) <= TOL[prec]


@pytest.mark.parametrize("nx,ny,prec", PLAN1_SHAPES)
def test_fft_plan1_matches_oracle(orc, gpu, monkeypatch, nx, ny, prec):
    """The alternative register-FFT radix plans (half the registers per thread),
    forced with LLG_B200_FFT_PLAN=1, against the oracle: fields and three RK45 steps."""
    monkeypatch.setenv("LLG_B200_FFT_PLAN", "1")
    c = case(nx, ny, dmi=2e-3, k_u=1e5)
    g = gpu_solver(gpu, c, prec)
    monkeypatch.delenv("LLG_B200_FFT_PLAN")
    rp, cp = g.fft_plans()
    assert cp // 2 == 1 and rp in (0, 1)
    o = oracle_solver(orc, c)
    m = random_m(orc, nx * ny, 13 + nx)
    g.set_state(m)
    bext = (0.01, 0.0, -0.02)
    p = gpu.LLGParams(GAMMA, 0.1, 1e-13, bext)
    assert rel_err(g.build_h_eff(p, 2), o.build_h_eff(m, bext, 2)) <= TOL[prec]
    assert rel_err(g.compute_demag_field(), o.demag_field(m)) <= TOL[prec]
    po = orc.make_params(GAMMA, 0.1, 1e-13, bext)
    mo = m.copy()
    for _ in range(3):
        ro = o.step_rk45(mo, po, 2, 1e-5, 0.8, 1e-19, 1e-11)
        rg = g.step_rk45(p, 2, 1e-5, 0.8, 1e-19, 1e-11)
        assert ro[1] == rg[1]
        p.dt = po.dt
    assert np.abs(g.get_state() - mo).max() <= (1e-12 if prec else 2e-6)
