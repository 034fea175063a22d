"""CPU tests of the oracle's restatement of the AMR demag consumers
(compute_coarse_fft_demag, coarse_fft_demag.rs:367-511; the AllFft branch of
AmrStepper::compute_demag, amr/stepper.rs:799-835), pinned by the reference's
own unit tests (coarse_fft_demag.rs:539-716) and by a pure-Python restatement
of the restriction and the bilinear sampler.  The cells are 5 x 5 x 2.5 nm
(the reference's tests use 1 nm thick cells): the properties are the same and the
FP64 kernel integration, whose point count grows with dx/dz, stays short."""
import math

import numpy as np
import pytest

import amr_cases as A


def _grid(orc, nx, ny, dx=A.DX, dy=A.DY, dz=A.DZ):
    return orc.make_grid(nx, ny, dx, dy, dz)


def _mat(orc, demag=True):
    return orc.make_material(A.MS, 0.0, demag=demag)


def _vortex_field(nx, ny, dx, dy):
    m = np.empty((nx * ny, 3))
    for j in range(ny):
        for i in range(nx):
            m[j * nx + i] = A.vortex((i + 0.5) * dx, (j + 0.5) * dy, nx * dx, ny * dy)
    return m


def test_validated_ratio_reference_cases(orc, gpu):
    # validated_ratio_rejects_bad_divisor / _too_small (coarse_fft_demag.rs:693-715)
    for (nx, ny, r, want) in [(30, 32, 4, 1), (32, 32, 4, 4), (7, 13, 1, 1), (8, 8, 4, 1), (16, 16, 4, 4)]:
        assert orc.validated_ratio(nx, ny, r) == want
        assert gpu.validated_ratio(nx, ny, r) == want


def test_coarsen_ratio_from_env(gpu, monkeypatch):
    for raw, want in [(None, 1), ("2", 2), (" 4 ", 4), ("3", 1), ("0", 1), ("x", 1), ("-2", 1)]:
        if raw is None:
            monkeypatch.delenv("LLG_DEMAG_COARSEN_RATIO", raising=False)
        else:
            monkeypatch.setenv("LLG_DEMAG_COARSEN_RATIO", raw)
        assert gpu.coarsen_ratio_from_env() == want


def test_zero_patches_reproduce_uniform_fft_exactly(orc):
    # zero_patches_reproduces_fft_exactly (coarse_fft_demag.rs:555-583)
    g = _grid(orc, 32, 32)
    m = _vortex_field(32, 32, A.DX, A.DY)
    bref = orc.Solver(g, _mat(orc)).demag_field(m)
    bc, bp = orc.coarse_fft_demag(g, _mat(orc), m, [])
    assert bp == []
    assert np.array_equal(bc, bref)


def test_restrict_l0_uniform_and_charge_cancellation(orc):
    # restrict_l0_to_demag_uniform_m / _charge_cancellation (coarse_fft_demag.rs:585-628)
    v = np.array([1.0, 0.0, 0.3]) / math.sqrt(1.09)
    out = orc.restrict_l0_to_demag_grid(4, np.tile(v, (16, 1)), 2, 2, 2)
    assert np.abs(out - v).max() < 1e-14
    m = np.array([[1.0, 0, 0], [-1.0, 0, 0], [1.0, 0, 0], [-1.0, 0, 0]])
    out = orc.restrict_l0_to_demag_grid(2, m, 1, 1, 2)
    assert np.abs(out).max() < 1e-14


def test_super_coarse_r2_accuracy(orc):
    # super_coarse_r2_accuracy (coarse_fft_demag.rs:630-691): RMSE / max|B| < 10 %
    g = _grid(orc, 64, 64)
    m = _vortex_field(64, 64, A.DX, A.DY)
    bref = orc.Solver(g, _mat(orc)).demag_field(m)
    b2, _ = orc.coarse_fft_demag(g, _mat(orc), m, [], ratio=2)
    bmax = np.linalg.norm(bref, axis=1).max()
    rmse = math.sqrt(np.mean(np.sum((bref - b2) ** 2, axis=1))) / bmax
    assert 0.0 < rmse < 0.10
    # R = 2 on this grid is the same as the explicit restrict -> FFT -> interpolate chain
    dm = orc.restrict_l0_to_demag_grid(64, m, 32, 32, 2)
    dg = _grid(orc, 32, 32, 2 * A.DX, 2 * A.DY)
    db = orc.Solver(dg, _mat(orc)).demag_field(dm)
    b_chain = np.array([orc.sample_bilinear(dg, db, (i + 0.5) * A.DX, (j + 0.5) * A.DY)
                        for j in range(64) for i in range(64)])
    assert np.array_equal(b2, b_chain)


def _py_sample(field, nx, ny, dx, dy, x, y):
    """sample_bilinear (amr/interp.rs:28-72) restated in Python."""
    fx, fy = x / dx - 0.5, y / dy - 0.5
    i0f, j0f = math.floor(fx), math.floor(fy)
    tx, ty = fx - i0f, fy - j0f
    cl = lambda i, n: min(max(i, 0), n - 1)
    i0, j0, i1, j1 = cl(int(i0f), nx), cl(int(j0f), ny), cl(int(i0f) + 1, nx), cl(int(j0f) + 1, ny)
    out = []
    for c in range(3):
        a = field[j0 * nx + i0][c] * (1.0 - tx) + field[j0 * nx + i1][c] * tx
        b = field[j1 * nx + i0][c] * (1.0 - tx) + field[j1 * nx + i1][c] * tx
        out.append(a * (1.0 - ty) + b * ty)
    return out


def _py_restrict(mc, patches):
    """restrict_m_to_coarse (coarse_fft_demag.rs:170-240) restated in Python."""
    out = mc.copy()
    for p in patches:
        for jc in range(p.cny):
            for ic in range(p.cnx):
                dst = (p.j0 + jc) * A.NX + p.i0 + ic
                if p.parent_material is not None and not p.parent_material[jc * p.cnx + ic]:
                    out[dst] = 0.0
                    continue
                s, n = [0.0, 0.0, 0.0], 0
                for fj in range(p.ratio):
                    for fi in range(p.ratio):
                        idx = (p.ghost + jc * p.ratio + fj) * p.pnx + p.ghost + ic * p.ratio + fi
                        if p.geom_mask_fine is not None and not p.geom_mask_fine[idx]:
                            continue
                        for c in range(3):
                            s[c] += float(p.m[idx][c])
                        n += 1
                if n == 0:
                    out[dst] = 0.0
                else:
                    inv = 1.0 / n
                    out[dst] = [s[0] * inv, s[1] * inv, s[2] * inv]
    return out


def test_restriction_and_sampling_match_python_restatement(orc):
    mc, patches = A.hierarchy()
    base = _grid(orc, A.NX, A.NY)
    enh = orc.restrict_m_to_coarse(base, mc, patches)
    assert np.array_equal(enh, _py_restrict(mc, patches))
    # the overlapping level-2 patch wins over the level-1 patch under it
    p1, p2, p3 = patches
    assert not np.array_equal(enh[12 * A.NX + 11], orc.restrict_m_to_coarse(base, mc, [p1])[12 * A.NX + 11])
    # parent cells without material are zero; unrefined cells keep the base value
    assert (p2.parent_material == 0).any()
    jc, ic = np.argwhere(p2.parent_material.reshape(p2.cny, p2.cnx) == 0)[0]
    assert not enh[(p2.j0 + jc) * A.NX + p2.i0 + ic].any()
    assert np.array_equal(enh[0], mc[0])
    # un-normalised: averages of unit vectors are shorter than 1
    assert np.linalg.norm(enh, axis=1).min() < 0.999
    # coarse-FFT patch samples = bilinear samples of the L0 field at the patch cell centres
    bc, bp = orc.coarse_fft_demag(base, _mat(orc), mc, patches)
    for p, b in zip(patches, bp):
        fdx, fdy = A.DX / p.ratio, A.DY / p.ratio
        for j in range(0, p.pny, 3):
            for i in range(0, p.pnx, 2):
                x = (p.i0 * p.ratio + (i - p.ghost) + 0.5) * fdx
                y = (p.j0 * p.ratio + (j - p.ghost) + 0.5) * fdy
                assert list(b[j * p.pnx + i]) == _py_sample(bc, A.NX, A.NY, A.DX, A.DY, x, y)
    # the L0 field is the uniform FFT demag of the restricted m
    assert np.array_equal(bc, orc.Solver(base, _mat(orc)).demag_field(enh))


def test_no_demag_gives_zero_and_no_patch_fields(orc):
    mc, patches = A.hierarchy()
    bc, bp = orc.coarse_fft_demag(_grid(orc, A.NX, A.NY), _mat(orc, demag=False), mc, patches)
    assert bp == [] and not bc.any()


def test_allfft_masks_and_samples(orc):
    fine = _grid(orc, 2 * A.NX, 2 * A.NY, A.DX / 2, A.DY / 2)
    base = _grid(orc, A.NX, A.NY)
    m = _vortex_field(2 * A.NX, 2 * A.NY, A.DX / 2, A.DY / 2)
    mask = np.ones(4 * A.NX * A.NY, dtype=np.uint8)
    mask[: 2 * A.NX * 5] = 0
    m[mask == 0] = 0.0
    bf, bc = orc.allfft_demag(fine, _mat(orc), m, mask, base)
    assert not bf[mask == 0].any()
    braw = orc.Solver(fine, _mat(orc)).demag_field(m)
    assert np.array_equal(bf[mask == 1], braw[mask == 1])
    for j in range(0, A.NY, 5):
        for i in range(0, A.NX, 3):
            want = _py_sample(bf, 2 * A.NX, 2 * A.NY, A.DX / 2, A.DY / 2, (i + 0.5) * A.DX, (j + 0.5) * A.DY)
            assert list(bc[j * A.NX + i]) == want


def test_benchmark_hierarchy_geometry(gpu):
    """The benchmark's AMR workload: patches inside the 192x192 base, fine m of unit
    vectors on each patch grid incl. ghosts, and the library's cell count per patch."""
    import workloads as W

    mc, patches = W.amr_vortex_hierarchy()
    assert mc.shape == (192 * 192, 3)
    assert np.allclose(np.linalg.norm(mc, axis=1), 1.0)
    cover = np.zeros((192, 192), dtype=int)
    for p in patches:
        assert p.i0 >= 0 and p.j0 >= 0 and p.i0 + p.cnx <= 192 and p.j0 + p.cny <= 192
        assert p.m.shape == (p.pnx * p.pny, 3) and np.allclose(np.linalg.norm(p.m, axis=1), 1.0)
        gp = gpu.AmrPatch(p.i0, p.j0, p.cnx, p.cny, p.ratio, p.ghost, p.m)
        assert gpu.lib().llg_amr_patch_cells(gpu.C.byref(gp._c())) == p.pnx * p.pny
        cover[p.j0:p.j0 + p.cny, p.i0:p.i0 + p.cnx] = 1
    assert 0.15 < cover.mean() < 0.17          # level-1 coverage of the quoted workload (~16 %)
    assert sorted({p.ratio for p in patches}) == [2, 4, 8]
