"""Shared case builders for the parity tests: one description, two engines."""
import numpy as np

GAMMA = 1.76085963023e11


def case(nx, ny, dx=4e-9, dy=4e-9, dz=3e-9, ms=8e5, a_ex=1.3e-11, k_u=0.0, easy=(0.0, 0.0, 1.0), dmi=None,
         demag=True, mask=None):
    return dict(nx=nx, ny=ny, dx=dx, dy=dy, dz=dz, ms=ms, a_ex=a_ex, k_u=k_u, easy=easy, dmi=dmi, demag=demag,
                mask=mask)


def oracle_solver(orc, c):
    g = orc.make_grid(c["nx"], c["ny"], c["dx"], c["dy"], c["dz"])
    m = orc.make_material(c["ms"], c["a_ex"], c["k_u"], c["easy"], c["dmi"], c["demag"])
    return orc.Solver(g, m, c["mask"])


def gpu_solver(L, c, precision):
    g = L.Grid2D(c["nx"], c["ny"], c["dx"], c["dy"], c["dz"])
    m = L.Material(c["ms"], c["a_ex"], c["k_u"], c["easy"], c["dmi"], c["demag"])
    return L.Solver(g, m, precision, c["mask"])


def random_m(orc, n, seed, mask=None):
    m = orc.init_random(n, seed)
    if mask is not None:
        m[np.asarray(mask).reshape(-1) == 0] = 0.0
    return m


def holes_mask(nx, ny, holes, dx=1.0, dy=1.0):
    """Film with circular holes: mask_disk_at semantics (geometry_mask.rs:336-373) inverted.

    holes: list of (cx, cy, r) in cells, centred coordinates."""
    msk = np.ones((ny, nx), dtype=np.uint8)
    for j in range(ny):
        for i in range(nx):
            x = (i + 0.5 - nx * 0.5) * dx
            y = (j + 0.5 - ny * 0.5) * dy
            for (cx, cy, r) in holes:
                if (x - cx * dx) ** 2 + (y - cy * dy) ** 2 <= (r * dx) ** 2:
                    msk[j, i] = 0
    return msk.reshape(-1)


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale
