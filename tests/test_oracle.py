"""CPU tests of the FP64 oracle: the reference's own known-answer tests, golden
fixtures (tests/golden/, pure-Python restatements) and independent numerics."""
import json
import math
import os

import numpy as np
import pytest

from helpers import GAMMA

HERE = os.path.dirname(os.path.abspath(__file__))
MU0 = 4.0 * math.pi * 1e-7


def test_fft_matches_numpy(orc):
    rng = np.random.default_rng(0)
    for n in [1, 2, 3, 4, 5, 7, 8, 12, 14, 22, 49, 64, 96, 121, 192, 384, 1000, 2048]:
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        ref = np.fft.fft(x)
        assert np.abs(orc.fft(x) - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())
        assert np.abs(orc.fft(x, inverse=True) - np.fft.ifft(x) * n).max() <= 1e-13 * max(1.0, np.abs(ref).max())


def test_xorshift_matches_golden(orc):
    gold = json.load(open(os.path.join(HERE, "golden", "xorshift_f64.json")))
    for seed, vals in gold.items():
        assert np.array_equal(orc.xorshift_f64(int(seed), len(vals)), np.array(vals))


def test_kernel_components_match_golden(orc):
    for e in json.load(open(os.path.join(HERE, "golden", "kernel_components.json"))):
        got = orc.kernel_components(*e["cell"], e["sx"], e["sy"])
        assert np.array_equal(got, np.array(e["k"])), e


def test_single_cube_cell_bz_is_minus_mu0_over_3(orc):
    # demag_fft_uniform.rs:1261-1293
    g = orc.make_grid(1, 1, 1.0, 1.0, 1.0)
    s = orc.Solver(g, orc.make_material(1.0, 0.0, demag=True))
    b = s.demag_field(np.array([[0.0, 0.0, 1.0]]))
    assert abs(b[0, 2] - (-MU0 / 3.0)) < 1e-3


def test_demag_2x2_uniform_z_symmetry(orc):
    # validation.rs:478-552
    g = orc.make_grid(2, 2, 1.0, 1.0, 1.0)
    s = orc.Solver(g, orc.make_material(1.0, 0.0, demag=True))
    m = np.tile([0.0, 0.0, 1.0], (4, 1))
    b = s.demag_field(m)
    assert np.abs(b[:, 0]).max() < 1e-10 and np.abs(b[:, 1]).max() < 1e-10
    assert b[:, 2].max() - b[:, 2].min() < 1e-10
    assert b[0, 2] < 0
    nzz = -b[0, 2] / MU0
    assert 0.05 < nzz < 1.05


def test_demag_2x2_nii_bounds(orc):
    # validation.rs:558-615
    g = orc.make_grid(2, 2, 1.0, 1.0, 1.0)
    s = orc.Solver(g, orc.make_material(1.0, 0.0, demag=True))
    n = []
    for c in range(3):
        m = np.zeros((4, 3))
        m[:, c] = 1.0
        n.append(-s.demag_field(m)[0, c] / MU0)
    assert all(0.0 < x < 1.2 for x in n)
    assert 0.5 < sum(n) < 2.5


def test_demag_energy_nonnegative_uniform(orc):
    # validation.rs:617-644
    g = orc.make_grid(32, 32, 5e-9, 5e-9, 1e-9)
    s = orc.Solver(g, orc.make_material(1.0, 0.0, demag=True))
    m = np.tile([0.0, 0.0, 1.0], (32 * 32, 1))
    assert s.energy(m, (0, 0, 0)).demag >= 0.0


def test_dmi_field_flips_sign_with_d(orc):
    # validation.rs:395-472
    nx = 9
    m = np.zeros((nx, 3))
    for i in range(nx):
        mz = min(max((i - (nx - 1) / 2) * 0.01, -0.2), 0.2)
        m[i] = [math.sqrt(1 - mz * mz), 0.0, mz]
    g = orc.make_grid(nx, 1, 1.0, 1.0, 1.0)
    bp = orc.Solver(g, orc.make_material(8e5, 13e-12, 0.0, dmi=1e-4)).build_h_eff(m, (0, 0, 0), 2)
    bm = orc.Solver(g, orc.make_material(8e5, 13e-12, 0.0, dmi=-1e-4)).build_h_eff(m, (0, 0, 0), 2)
    assert abs(bp[4, 0]) > 0
    assert abs(bp[4, 0] + bm[4, 0]) < 1e-10 * max(abs(bp[4, 0]), 1.0)


def neel_wall(nx, ny, dx, x0, width):
    # init_neel_wall_x (vector_field.rs:103-127), used by init_bloch_wall (:162)
    m = np.zeros((ny * nx, 3))
    for j in range(ny):
        for i in range(nx):
            u = ((i + 0.5) * dx - x0) / width
            mz, mx = math.tanh(u), 1.0 / math.cosh(u)
            nrm = math.sqrt(mx * mx + mz * mz)
            m[j * nx + i] = [mx / nrm, 0.0, mz / nrm]
    return m


def test_energy_gradient_consistency(orc):
    # validation.rs:222-318: dE ~ -Ms V B.dm within 5 %
    g = orc.make_grid(16, 16, 5e-9, 5e-9, 5e-9)
    mat = orc.make_material(8e5, 13e-12, 500.0, (0, 0, 1))
    s = orc.Solver(g, mat)
    m = neel_wall(16, 16, 5e-9, 0.5 * 16 * 5e-9, 5 * 5e-9)
    b = s.build_h_eff(m, (0, 0, 0), 2)
    e0 = s.energy(m, (0, 0, 0))
    idx = 8 * 16 + 8
    m0 = m[idx]
    a = np.array([0.37, -0.24, 0.91])
    d = a - np.dot(m0, a) * m0
    d /= np.linalg.norm(d)
    m1 = m0 + 1e-6 * d
    m1 /= np.linalg.norm(m1)
    mp = m.copy()
    mp[idx] = m1
    e1 = s.energy(mp, (0, 0, 0))
    de = (e1.exchange + e1.anisotropy + e1.zeeman + e1.dmi + e1.demag) - (
        e0.exchange + e0.anisotropy + e0.zeeman + e0.dmi + e0.demag)
    pred = -8e5 * (5e-9) ** 3 * np.dot(b[idx], m1 - m0)
    scale = 8e5 * (5e-9) ** 3 * np.linalg.norm(b[idx]) * 1e-6
    assert abs(de - pred) < 5e-2 * scale


def test_rk45_macrospin_quarter_turn(orc):
    # validation.rs:646-745, plus the analytic phase check
    g = orc.make_grid(1, 1, 1.0, 1.0, 1.0)
    s = orc.Solver(g, orc.make_material(8e5, 0.0, 0.0))
    m = np.array([[1.0, 0.0, 0.0]])
    b0 = 0.1
    p = orc.make_params(GAMMA, 0.0, 1e-14, (0.0, 0.0, b0))
    t_target = (math.pi / 2) / (GAMMA * b0)
    t = 0.0
    attempts = 0
    while t < t_target:
        attempts += 1
        assert attempts < 200000
        p.dt = min(p.dt, t_target - t)
        eps, acc, dtu = s.step_rk45(m, p, 2, 1e-5, 0.8, 1e-18, 1e-11)
        if acc:
            t += dtu
    v = m[0]
    assert abs(v[2]) < 0.1 and abs(v[1]) > 0.9 and abs(v[0]) < 0.3
    # dm/dt = -gamma m x B with x cross z = -y: +x precesses to +y for B along +z
    assert abs(v[1] - 1.0) < 1e-5 and abs(v[0]) < 1e-5


def test_fft_demag_equals_direct_convolution(orc):
    for (nx, ny) in [(1, 1), (3, 5), (7, 4), (12, 10)]:
        g = orc.make_grid(nx, ny, 5e-9, 4e-9, 3e-9)
        s = orc.Solver(g, orc.make_material(8e5, 1.3e-11, demag=True))
        m = orc.init_random(nx * ny, 17 + nx)
        b1 = s.demag_field(m)
        b2 = orc.demag_field_direct(g, 8e5, m)
        assert np.abs(b1 - b2).max() <= 1e-12 * np.abs(b2).max()


def test_kernel_spectrum_is_real_and_even(orc):
    nx, ny = 6, 5
    g = orc.make_grid(nx, ny, 4e-9, 4e-9, 3e-9)
    s = orc.Solver(g, orc.make_material(8e5, 1.3e-11, demag=True))
    k = s.kernel_kspace()
    for c in range(4):
        assert np.abs(k[c].imag).max() <= 1e-12 * np.abs(k[c].real).max()
    px, py = 2 * nx, 2 * ny
    kx = (px - np.arange(px)) % px
    ky = (py - np.arange(py)) % py
    for c, sgn in [(0, 1), (2, 1), (3, 1)]:
        assert np.allclose(k[c].real, k[c].real[:, kx], rtol=0, atol=1e-15)
        assert np.allclose(k[c].real, k[c].real[ky, :], rtol=0, atol=1e-15)
    assert np.allclose(k[1].real, -k[1].real[:, kx], rtol=0, atol=1e-15)
    assert np.allclose(k[1].real, -k[1].real[ky, :], rtol=0, atol=1e-15)


def test_relax_reaches_torque_threshold(orc):
    g = orc.make_grid(16, 16, 5e-9, 5e-9, 5e-9)
    s = orc.Solver(g, orc.make_material(8e5, 13e-12, 500.0, (0, 0, 1)))
    m = np.tile([0.05, 0.0, math.sqrt(1 - 0.05 ** 2)], (256, 1))
    p = orc.make_params(GAMMA, 0.5, 2e-13, (0.0, 0.0, 1e-6))
    st = orc.default_relax_settings(torque_threshold=1e-6)
    rep = s.relax(m, p, 0, st)
    assert rep.stop_reason == 2  # TightenFloorReached
    assert rep.has_final_torque_max and rep.final_torque_max <= 1e-6
    assert m[:, 2].min() > 0.999


def test_init_states(orc):
    m = orc.init_random(100, 3)
    assert np.allclose(np.linalg.norm(m, axis=1), 1.0)
    x = orc.xorshift_f64(3, 300).reshape(100, 3) * 2 - 1
    assert np.allclose(m, x / np.linalg.norm(x, axis=1, keepdims=True), rtol=0, atol=1e-15)
    base = np.ones((10, 3))
    base[4] = 0
    w = orc.init_uniform_with_noise(10, (1, 0, 0), 0.05, 9, base)
    assert np.all(w[4] == 0) and np.allclose(np.linalg.norm(np.delete(w, 4, 0), axis=1), 1.0)
