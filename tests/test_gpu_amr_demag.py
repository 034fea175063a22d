"""The AMR consumers of the uniform FFT demag on the GPU (llg_coarse_fft_demag,
llg_amr_restrict_m, llg_amr_allfft_demag) against the FP64 oracle.

Restriction and sampling keep the reference's operation order without
contraction, so given the same input they match the oracle bit for bit; the FFT
demag in between matches to FP64 round-off: the GPU integrates the demag kernel
with the same rule but sums the integration points in another order, which
leaves relative differences of 1e-11 (5 nm cells) to 2e-10 (20 x 20 x 2.5 nm
cells of the R = 4 demag grid); the tolerance is 1e-9."""
import numpy as np
import pytest

import amr_cases as A

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _objs(gpu, orc, nx=A.NX, ny=A.NY, dx=A.DX, dy=A.DY, demag=True):
    return (gpu.Grid2D(nx, ny, dx, dy, A.DZ), orc.make_grid(nx, ny, dx, dy, A.DZ),
            gpu.Material(A.MS, 0.0, demag=demag), orc.make_material(A.MS, 0.0, demag=demag))


def _gpu_patches(gpu, patches):
    return [gpu.AmrPatch(p.i0, p.j0, p.cnx, p.cny, p.ratio, p.ghost, p.m, p.geom_mask_fine, p.parent_material)
            for p in patches]


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_restrict_m_bit_exact(gpu, orc):
    mc, patches = A.hierarchy()
    gg, og, _, _ = _objs(gpu, orc)
    h = gpu.AmrDemag(gg)
    out = h.restrict_m(mc, _gpu_patches(gpu, patches))
    assert np.array_equal(out, orc.restrict_m_to_coarse(og, mc, patches))
    # no patches: the base field itself
    assert np.array_equal(h.restrict_m(mc, []), mc)


@pytest.mark.parametrize("ratio", [1, 2, 4])
def test_coarse_fft_demag_matches_oracle(gpu, orc, ratio):
    mc, patches = A.hierarchy()
    gg, og, gm, om = _objs(gpu, orc)
    h = gpu.AmrDemag(gg, coarsen_ratio=ratio)
    assert h.ratio == ratio
    bc, bp = h.compute(gm, mc, _gpu_patches(gpu, patches))
    oc, op = orc.coarse_fft_demag(og, om, mc, patches, ratio=ratio)
    assert _rel(bc, oc) < TOL
    assert len(bp) == len(op) == 3
    for p, b, o in zip(patches, bp, op):
        assert b.shape == (p.pnx * p.pny, 3)
        assert _rel(b, o) < TOL
        # the patch samples are the oracle's bilinear samples of the GPU's own L0 field
        fdx, fdy = A.DX / p.ratio, A.DY / p.ratio
        for j in range(0, p.pny, 3):
            for i in range(0, p.pnx, 2):
                x = (p.i0 * p.ratio + (i - p.ghost) + 0.5) * fdx
                y = (p.j0 * p.ratio + (j - p.ghost) + 0.5) * fdy
                assert np.array_equal(b[j * p.pnx + i], orc.sample_bilinear(og, bc, x, y))


def test_invalid_ratios_fall_back_to_one(gpu, orc):
    gg, _, _, _ = _objs(gpu, orc)
    for r in (3, 6, 16, 64, 0):   # not a power of two, or fewer than 4 cells left, or < 1
        assert gpu.AmrDemag(gg, coarsen_ratio=r).ratio == 1


def test_zero_patches_equal_uniform_demag(gpu, orc):
    mc, _ = A.hierarchy()
    gg, og, gm, om = _objs(gpu, orc)
    bc, bp = gpu.AmrDemag(gg).compute(gm, mc, [])
    assert bp == []
    # the uniform demag of the same grid through the stand-alone operator
    op = gpu.DemagOp(gg)
    assert np.array_equal(bc, op.field(A.MS, mc))
    assert _rel(bc, orc.Solver(og, om).demag_field(mc)) < TOL


def test_no_demag(gpu, orc):
    mc, patches = A.hierarchy()
    gg, _, gm, _ = _objs(gpu, orc, demag=False)
    bc, bp = gpu.AmrDemag(gg).compute(gm, mc, _gpu_patches(gpu, patches))
    assert bp == [] and not bc.any()


def test_repeated_calls_with_changing_patch_sets(gpu, orc):
    """Buffers grow and are reused across calls with different patch lists."""
    mc, patches = A.hierarchy()
    gg, og, gm, om = _objs(gpu, orc)
    h = gpu.AmrDemag(gg)
    for sub in ([patches[0]], patches, [patches[2], patches[1]], []):
        bc, bp = h.compute(gm, mc, _gpu_patches(gpu, sub))
        oc, op = orc.coarse_fft_demag(og, om, mc, sub)
        assert _rel(bc, oc) < TOL
        for b, o in zip(bp, op):
            assert _rel(b, o) < TOL


def test_allfft_matches_oracle(gpu, orc):
    fine_g, fine_o, gm, om = _objs(gpu, orc, 2 * A.NX, 2 * A.NY, A.DX / 2, A.DY / 2)
    base_g, base_o, _, _ = _objs(gpu, orc)
    m = np.array([A.vortex((i + 0.5) * A.DX / 2, (j + 0.5) * A.DY / 2, A.NX * A.DX, A.NY * A.DY)
                  for j in range(2 * A.NY) for i in range(2 * A.NX)])
    mask = np.ones(4 * A.NX * A.NY, dtype=np.uint8)
    mask[: 2 * A.NX * 5] = 0
    m[mask == 0] = 0.0
    op = gpu.DemagOp(fine_g)
    bf, bc = gpu.allfft_demag(op, gm, m, mask, base_g)
    of, oc = orc.allfft_demag(fine_o, om, m, mask, base_o)
    assert not bf[mask == 0].any()
    assert _rel(bf, of) < TOL
    assert _rel(bc, oc) < TOL
    for j in range(0, A.NY, 3):
        for i in range(0, A.NX, 2):
            assert np.array_equal(bc[j * A.NX + i],
                                  orc.sample_bilinear(fine_o, bf, (i + 0.5) * A.DX, (j + 0.5) * A.DY))
    # a periodic operator is refused (the AllFft demag uses open boundaries)
    with pytest.raises(gpu.LLGError):
        gpu.allfft_demag(gpu.DemagOp(fine_g, pbc_x=2), gm, m, mask, base_g)


def test_allfft_device_entry_equals_host_entry(gpu):
    """llg_amr_allfft_demag_device on resident arrays gives the host entry's bits."""
    import torch

    import workloads as W

    nx = ny = 48
    mf = W.amr_fine_vortex(4 * nx, 4 * ny, 4e-9 / 4, 4e-9 / 4)
    fg = gpu.Grid2D(4 * nx, 4 * ny, 1e-9, 1e-9, 3e-9)
    bg = gpu.Grid2D(nx, ny, 4e-9, 4e-9, 3e-9)
    mat = gpu.Material(8e5, 1.3e-11, demag=True)
    op = gpu.DemagOp(fg)
    mask = np.ones(fg.nx * fg.ny, dtype=np.uint8)
    mask[: fg.nx * 5] = 0
    bf, bc = gpu.allfft_demag(op, mat, mf, mask, bg)
    d_m = torch.from_numpy(np.ascontiguousarray(mf)).cuda()
    d_k = torch.from_numpy(mask).cuda()
    d_bf = torch.empty_like(d_m)
    d_bc = torch.empty((nx * ny, 3), dtype=torch.float64, device="cuda")
    gpu.allfft_demag_device(op, mat, d_m.data_ptr(), d_k.data_ptr(), bg, d_bf.data_ptr(), d_bc.data_ptr(),
                            torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(d_bf.cpu().numpy(), bf)
    assert np.array_equal(d_bc.cpu().numpy(), bc)
    op.close()
