"""A small AMR hierarchy for the coarse-FFT / AllFft demag tests: a 32x32 base
grid holding a vortex, two level-1 patches (ratio 2, ghost 2; one with a fine
geometry mask and the parent_material flags derived from it) and one level-2
patch (ratio 4) overlapping the first, listed in the reference's processing
order (level 1, then level 2)."""
import math

import numpy as np

NX, NY, DX, DY, DZ, MS = 32, 32, 5e-9, 5e-9, 2.5e-9, 8.0e5


def vortex(x, y, lx, ly):
    """normalize([-y/r, x/r, 0.3]) at centred, domain-scaled coordinates (the
    make_vortex_m state of coarse_fft_demag.rs's tests, evaluated at a point)."""
    xr, yr = x / lx - 0.5, y / ly - 0.5
    r = max(math.hypot(xr, yr), 1e-12)
    v = np.array([-yr / r, xr / r, 0.3])
    return v / np.linalg.norm(v)


class Patch:
    def __init__(self, i0, j0, cnx, cny, ratio, ghost, m, geom_mask_fine=None, parent_material=None):
        self.i0, self.j0, self.cnx, self.cny, self.ratio, self.ghost = i0, j0, cnx, cny, ratio, ghost
        self.pnx, self.pny = cnx * ratio + 2 * ghost, cny * ratio + 2 * ghost
        self.m, self.geom_mask_fine, self.parent_material = m, geom_mask_fine, parent_material


def _fine_patch(i0, j0, cnx, cny, ratio, ghost, rng, hole=None):
    lx, ly = NX * DX, NY * DY
    pnx, pny = cnx * ratio + 2 * ghost, cny * ratio + 2 * ghost
    fdx, fdy = DX / ratio, DY / ratio
    m = np.empty((pny * pnx, 3))
    mask = np.ones(pny * pnx, dtype=np.uint8)
    for j in range(pny):
        for i in range(pnx):
            x = (i0 * ratio + (i - ghost) + 0.5) * fdx
            y = (j0 * ratio + (j - ghost) + 0.5) * fdy
            v = vortex(x, y, lx, ly) + 0.05 * rng.standard_normal(3)
            m[j * pnx + i] = v / np.linalg.norm(v)
            if hole is not None and (x - hole[0]) ** 2 + (y - hole[1]) ** 2 <= hole[2] ** 2:
                mask[j * pnx + i] = 0
    if hole is None:
        return Patch(i0, j0, cnx, cny, ratio, ghost, m)
    parent = np.zeros(cny * cnx, dtype=np.uint8)
    for jc in range(cny):
        for ic in range(cnx):
            blk = [mask[(ghost + jc * ratio + fj) * pnx + ghost + ic * ratio + fi]
                   for fj in range(ratio) for fi in range(ratio)]
            parent[jc * cnx + ic] = 1 if any(blk) else 0
    return Patch(i0, j0, cnx, cny, ratio, ghost, m, mask, parent)


def hierarchy(seed=3):
    """(base m [NX*NY, 3], [patches]) with the patches in processing order."""
    rng = np.random.default_rng(seed)
    lx, ly = NX * DX, NY * DY
    mc = np.empty((NX * NY, 3))
    for j in range(NY):
        for i in range(NX):
            mc[j * NX + i] = vortex((i + 0.5) * DX, (j + 0.5) * DY, lx, ly)
    p1 = _fine_patch(8, 10, 10, 8, 2, 2, rng)
    # a disk of vacuum around (23, 7) base cells: fully empty parents give zero
    p2 = _fine_patch(20, 4, 6, 6, 2, 2, rng, hole=(23.0 * DX, 7.0 * DY, 1.6 * DX))
    p3 = _fine_patch(11, 12, 4, 3, 4, 2, rng)
    return mc, [p1, p2, p3]
