"""Synthetic inputs of the benchmark workloads (host side, numpy).

Every workload is fully determined by its seed, so the same arrays feed the GPU
library and any CPU restatement.  Sizes and value ranges:

* ``film_128x32_relax_then_field`` — 128x32x1 film, 4x4x3 nm cells, Ms 8.0e5 A/m,
  A 1.3e-11 J/m, no anisotropy or DMI, demag on (open boundaries), alpha 0.02.
  m0 = +x with a Gaussian tilt of sigma 0.05 rad.  Relax with the settings of the
  reference's SP4 driver (st_problems/sp4.rs:164-235: RK23, max |m x B| 1e-4 T,
  max_err 1e-5, headroom 0.8, dt0 5e-14, dt 1e-18 .. 1e-11, energy stride 3 with
  tolerance 1e-12, no plateau test, floor 1e-9, at most 2e6 steps), then 1 ns of
  RK45 (max_err 1e-6, headroom 0.8, dt0 1e-13, dt 1e-19 .. 1e-11, sp4.rs:159-167)
  under 20 mT in-plane at a seeded angle, with <m> sampled every 10 ps and dt
  clamped onto each sample time as sp4.rs:306-333 does.
* ``film_1024_dmi`` — 1024x1024x1 film, 2 nm cubes, Ms 5.8e5, A 1.5e-11, Ku 8e5
  along +z, interfacial D 3e-3 J/m^2, alpha 0.3, random m0 (init_random,
  initial_states.rs:59-68, seed 1), demag on; RK45 with max_err 1e-5.
* ``mixed_film_batch`` — n films (256 by default) with nx in {64,96,128,192,256},
  ny in {32,64,128}, 4x4x3 nm cells, Ms U[6e5,9e5], A U[1e-11,1.5e-11],
  alpha 0.02, in-plane field 0-50 mT at a seeded angle, m0 = +x with 0.1 noise
  (init_uniform_with_noise, initial_states.rs:43-56); FP32 RK45 max_err 1e-5,
  per-film dt, 1 ns each.
* ``holey_film_batch`` — n films of size x size (128 or 256), 4x4x3 nm cells,
  Ms 8e5, A 1.3e-11, D U[0,2e-3], 0-6 circular holes of radius 8-24 cells
  (mask_disk_at semantics, geometry_mask.rs:336-373, cell centres measured from
  the film centre), random unit m0 with zero in the holes, in-plane field
  0-30 mT; relaxed to max torque 1e-6 T.
"""
import math

import numpy as np

GAMMA = 1.76085963023e11   # params.rs:16


class Film:
    """One film of a workload: geometry, material, optional mask, field and m0."""

    def __init__(self, nx, ny, dx, dy, dz, ms, a_ex, k_u=0.0, easy=(0.0, 0.0, 1.0), dmi=None, demag=True,
                 mask=None, b_ext=(0.0, 0.0, 0.0), m0=None, alpha=0.02):
        self.nx, self.ny, self.dx, self.dy, self.dz = int(nx), int(ny), dx, dy, dz
        self.ms, self.a_ex, self.k_u, self.easy, self.dmi, self.demag = ms, a_ex, k_u, tuple(easy), dmi, demag
        self.mask, self.b_ext, self.m0, self.alpha = mask, tuple(b_ext), m0, alpha

    @property
    def n(self):
        return self.nx * self.ny

    def grid(self, L):
        return L.Grid2D(self.nx, self.ny, self.dx, self.dy, self.dz)

    def material(self, L):
        return L.Material(self.ms, self.a_ex, self.k_u, self.easy, self.dmi, self.demag)


def xorshift64(seed):
    """XorShift64 of initial_states.rs:230-254 as a generator of f64 in [0, 1)."""
    s = seed if seed else 0x9E3779B97F4A7C15
    mask = (1 << 64) - 1
    while True:
        s ^= (s << 13) & mask
        s ^= s >> 7
        s ^= (s << 17) & mask
        yield (s >> 11) * (1.0 / (1 << 53))


def gaussian_tilt(n, sigma, seed):
    """m = normalize(+x + sigma*(g1*y + g2*z)), g1, g2 standard normal by Box-Muller over XorShift64."""
    r = xorshift64(seed)
    m = np.empty((n, 3))
    two_pi = 2.0 * math.pi
    for i in range(n):
        g = [0.0, 0.0]
        for q in range(2):
            u1, u2 = next(r), next(r)
            g[q] = math.sqrt(-2.0 * math.log(1.0 - u1)) * math.cos(two_pi * u2)
        vx, vy, vz = 1.0, sigma * g[0], sigma * g[1]
        inv = 1.0 / math.sqrt(vx * vx + vy * vy + vz * vz)
        m[i] = (vx * inv, vy * inv, vz * inv)
    return m


def disk_holes_mask(nx, ny, dx, dy, holes):
    """Film mask with circular holes [(cx, cy, r)] in metres, centred cell coordinates."""
    i = np.arange(nx)
    j = np.arange(ny)
    x = (i + 0.5 - nx * 0.5) * dx
    y = (j + 0.5 - ny * 0.5) * dy
    X, Y = np.meshgrid(x, y)
    keep = np.ones((ny, nx), dtype=bool)
    for (cx, cy, r) in holes:
        ddx = X - cx
        ddy = Y - cy
        keep &= ~(ddx * ddx + ddy * ddy <= r * r)
    return keep.astype(np.uint8).reshape(-1)


# ---------------------------------------------------------------------------------------------

def film_128x32_relax_then_field(seed=11):
    rng = np.random.default_rng(seed)
    ang = float(rng.uniform(0.0, 2.0 * math.pi))
    f = Film(128, 32, 4e-9, 4e-9, 3e-9, 8.0e5, 1.3e-11, demag=True,
             b_ext=(0.02 * math.cos(ang), 0.02 * math.sin(ang), 0.0), alpha=0.02)
    f.m0 = gaussian_tilt(f.n, 0.05, seed)
    relax = dict(alpha=0.02, dt0=5e-14, torque_threshold=1e-4, max_err=1e-5, headroom=0.8, dt_min=1e-18,
                 dt_max=1e-11, energy_stride=3, rel_energy_tol=1e-12, torque_check_stride=1,
                 torque_plateau_checks=0, tighten_floor=1e-9, max_accepted_steps=2000000)
    run = dict(alpha=0.02, dt0=1e-13, max_err=1e-6, headroom=0.8, dt_min=1e-19, dt_max=1e-11, t_total=1e-9,
               dt_out=1e-11)
    return f, relax, run


def film_1024_dmi(nx=1024, ny=1024, seed=1):
    f = Film(nx, ny, 2e-9, 2e-9, 2e-9, 5.8e5, 1.5e-11, k_u=8e5, easy=(0.0, 0.0, 1.0), dmi=3e-3, demag=True,
             alpha=0.3)
    run = dict(dt0=1e-13, max_err=1e-5, headroom=0.8, dt_min=1e-18, dt_max=1e-11)
    return f, seed, run


def mixed_film_batch(n=256, seed=3):
    """Returns (films, run settings); m0 is filled by the caller's init_uniform_with_noise(seed + i)."""
    rng = np.random.default_rng(seed)
    nxs = [64, 96, 128, 192, 256]
    nys = [32, 64, 128]
    films = []
    for _ in range(n):
        nx = nxs[int(rng.integers(len(nxs)))]
        ny = nys[int(rng.integers(len(nys)))]
        ms = float(rng.uniform(6e5, 9e5))
        a = float(rng.uniform(1.0e-11, 1.5e-11))
        b = float(rng.uniform(0.0, 0.05))
        ang = float(rng.uniform(0.0, 2.0 * math.pi))
        films.append(Film(nx, ny, 4e-9, 4e-9, 3e-9, ms, a, demag=True,
                          b_ext=(b * math.cos(ang), b * math.sin(ang), 0.0), alpha=0.02))
    run = dict(dt0=1e-13, max_err=1e-5, headroom=0.8, dt_min=1e-18, dt_max=1e-11, t_total=1e-9, noise=0.1)
    return films, run


def holey_film_batch(n, size=128, seed=5):
    """Films with 0-6 holes; m0 is filled by the caller's init_random(seed*1000 + i) with holes zeroed."""
    rng = np.random.default_rng(seed)
    d = 4e-9
    films = []
    for _ in range(n):
        nh = int(rng.integers(0, 7))
        holes = []
        for _ in range(nh):
            r = float(rng.uniform(8, 24)) * d
            cx = float(rng.uniform(-0.5, 0.5)) * size * d
            cy = float(rng.uniform(-0.5, 0.5)) * size * d
            holes.append((cx, cy, r))
        mask = disk_holes_mask(size, size, d, d, holes)
        dmi = float(rng.uniform(0.0, 2e-3))
        b = float(rng.uniform(0.0, 0.03))
        ang = float(rng.uniform(0.0, 2.0 * math.pi))
        films.append(Film(size, size, d, d, 3e-9, 8e5, 1.3e-11, dmi=dmi, demag=True, mask=mask,
                          b_ext=(b * math.cos(ang), b * math.sin(ang), 0.0), alpha=0.5))
    relax = dict(dt0=1e-13, torque_threshold=1e-6, max_err=1e-5, headroom=0.8, dt_min=1e-18, dt_max=1e-11)
    return films, relax


# ---------------------------------------------------------------------------------------------

class AmrPatchSpec:
    """One patch of an AMR hierarchy (Patch2D, amr/patch.rs:15-80, as the demag
    consumers read it)."""

    def __init__(self, i0, j0, cnx, cny, ratio, ghost, m, geom_mask_fine=None, parent_material=None):
        self.i0, self.j0, self.cnx, self.cny, self.ratio, self.ghost = i0, j0, cnx, cny, ratio, ghost
        self.pnx, self.pny = cnx * ratio + 2 * ghost, cny * ratio + 2 * ghost
        self.m, self.geom_mask_fine, self.parent_material = m, geom_mask_fine, parent_material


def vortex_field(xs, ys, lx, ly):
    """m = normalize([-y/r, x/r, 0.3]) at centred, domain-scaled coordinates
    (the vortex of coarse_fft_demag.rs's tests), vectorised over points."""
    xr, yr = xs / lx - 0.5, ys / ly - 0.5
    r = np.maximum(np.hypot(xr, yr), 1e-12)
    v = np.stack([-yr / r, xr / r, np.full_like(xr, 0.3)], axis=-1)
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def amr_vortex_hierarchy(nx=192, ny=192, dx=4e-9, dy=4e-9, dz=3e-9, seed=13):
    """The coarse-FFT demag workload: a vortex in a nx x ny film of dx x dy x dz cells
    (Ms 8e5), refined around the core by level-1 patches (ratio 2, four 38x38 blocks,
    15.7 % of the film), level-2 patches (ratio 4, two 19x19 blocks) and one level-3
    patch (ratio 8, 12x12), ghost 2, fine m = the vortex plus 2 % seeded noise.  The
    AllFft equivalent is the film at 8x resolution (nx*8 x ny*8, dx/8 x dy/8 x dz),
    the 1536 x 1536 fine grid of coarse_fft_demag.rs:28-31 for the defaults.
    Returns (m_coarse [nx*ny, 3], patches in processing order)."""
    rng = np.random.default_rng(seed)
    lx, ly = nx * dx, ny * dy
    i = np.arange(nx)
    j = np.arange(ny)
    X, Y = np.meshgrid((i + 0.5) * dx, (j + 0.5) * dy)
    mc = vortex_field(X, Y, lx, ly).reshape(-1, 3)
    cx, cy = nx // 2, ny // 2
    rects = [(cx - 38, cy - 38, 38, 38, 2), (cx, cy - 38, 38, 38, 2), (cx - 38, cy, 38, 38, 2), (cx, cy, 38, 38, 2),
             (cx - 19, cy - 19, 19, 19, 4), (cx, cy, 19, 19, 4), (cx - 6, cy - 6, 12, 12, 8)]
    patches = []
    for (i0, j0, cnx, cny, r) in rects:
        g = 2
        pnx, pny = cnx * r + 2 * g, cny * r + 2 * g
        fi = np.arange(pnx)
        fj = np.arange(pny)
        FX, FY = np.meshgrid((i0 * r + (fi - g) + 0.5) * (dx / r), (j0 * r + (fj - g) + 0.5) * (dy / r))
        v = vortex_field(FX, FY, lx, ly).reshape(-1, 3) + 0.02 * rng.standard_normal((pnx * pny, 3))
        patches.append(AmrPatchSpec(i0, j0, cnx, cny, r, g, v / np.linalg.norm(v, axis=1, keepdims=True)))
    return mc, patches


def amr_fine_vortex(nx, ny, dx, dy):
    """The vortex on a uniform fine grid (the flattened hierarchy of the AllFft demag)."""
    X, Y = np.meshgrid((np.arange(nx) + 0.5) * dx, (np.arange(ny) + 0.5) * dy)
    return vortex_field(X, Y, nx * dx, ny * dy).reshape(-1, 3)


def film_cost(f):
    """Work estimate of one film per step: cells plus its padded transforms,
    2nx x 2ny x log2(2nx x 2ny) (the demag FFTs dominate)."""
    px, py = 2 * f.nx, 2 * f.ny
    return float(f.n) + float(px * py) * math.log2(max(px * py, 2))


def partition_films(films, world, rank):
    """Indices of the films rank `rank` of `world` advances: greedy longest-first
    assignment to the least-loaded rank (ties to the lower rank), so every film is
    taken by exactly one rank and loads are balanced by film_cost."""
    order = sorted(range(len(films)), key=lambda i: (-film_cost(films[i]), i))
    load = [0.0] * world
    owner = [0] * len(films)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += film_cost(films[i])
    return [i for i in range(len(films)) if owner[i] == rank]

