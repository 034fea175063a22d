"""ctypes wrapper of liboracle.so (CPU FP64 restatement; test infrastructure only)."""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

FIELD_EXCH_ANIS, FIELD_EXCH_ANIS_DMI, FIELD_FULL = 0, 1, 2
TORQUE_MAX, TORQUE_MEAN, TORQUE_RMS, TORQUE_MEANSQ = 0, 1, 2, 3


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int64), ("ny", C.c_int64), ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double)]


class Material(C.Structure):
    _fields_ = [("ms", C.c_double), ("a_ex", C.c_double), ("k_u", C.c_double), ("easy_axis", C.c_double * 3),
                ("dmi", C.c_double), ("has_dmi", C.c_int32), ("demag", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("gamma", C.c_double), ("alpha", C.c_double), ("dt", C.c_double), ("b_ext", C.c_double * 3)]


class RelaxSettings(C.Structure):
    _fields_ = [("max_err", C.c_double), ("headroom", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double),
                ("phase1_enabled", C.c_int32), ("phase2_enabled", C.c_int32), ("energy_stride", C.c_int64),
                ("rel_energy_tol", C.c_double), ("torque_metric", C.c_int32), ("has_torque_threshold", C.c_int32),
                ("torque_threshold", C.c_double), ("torque_check_stride", C.c_int64),
                ("torque_plateau_rel", C.c_double), ("torque_plateau_abs", C.c_double),
                ("torque_plateau_checks", C.c_int64), ("torque_plateau_min_checks", C.c_int64),
                ("tighten_factor", C.c_double), ("tighten_floor", C.c_double), ("max_accepted_steps", C.c_int64),
                ("has_final_torque_gate", C.c_int32), ("has_final_torque_gate_max", C.c_int32),
                ("final_torque_gate", C.c_double), ("final_torque_gate_max", C.c_double),
                ("gate_max_extra_accepted_steps", C.c_int64), ("gate_plateau_fails", C.c_int64)]


class RelaxReport(C.Structure):
    _fields_ = [("accepted_steps", C.c_int64), ("rejected_steps", C.c_int64), ("torque_checks", C.c_int64),
                ("torque_field_rebuilds", C.c_int64), ("stop_reason", C.c_int32), ("last_stage_stop", C.c_int32),
                ("has_final_torque", C.c_int32), ("has_final_torque_max", C.c_int32),
                ("final_torque", C.c_double), ("final_torque_max", C.c_double),
                ("final_max_err", C.c_double), ("final_dt", C.c_double)]


class MinimizeSettings(C.Structure):
    _fields_ = [("torque_threshold", C.c_double), ("max_iters", C.c_int64), ("lambda0", C.c_double),
                ("lambda_min", C.c_double), ("lambda_max", C.c_double), ("grow", C.c_double), ("shrink", C.c_double),
                ("stall_iters", C.c_int64), ("stall_rel", C.c_double), ("min_iters_before_stall", C.c_int64),
                ("has_dm_stop", C.c_int32), ("has_dm_torque_gate", C.c_int32),
                ("has_dm_torque_gate_max", C.c_int32), ("reserved", C.c_int32), ("dm_stop", C.c_double),
                ("dm_samples", C.c_int64), ("dm_torque_gate", C.c_double), ("dm_torque_gate_max", C.c_double),
                ("dm_min_iters", C.c_int64)]


class MinimizeReport(C.Structure):
    _fields_ = [("iters", C.c_int64), ("converged", C.c_int32), ("stalled", C.c_int32),
                ("dm_converged", C.c_int32), ("reserved", C.c_int32), ("final_torque", C.c_double),
                ("final_max_dm", C.c_double), ("final_tmean", C.c_double), ("final_lambda", C.c_double)]


class AmrPatch(C.Structure):
    _fields_ = [("i0", C.c_int64), ("j0", C.c_int64), ("cnx", C.c_int64), ("cny", C.c_int64),
                ("ratio", C.c_int64), ("ghost", C.c_int64), ("m", C.c_void_p), ("geom_mask_fine", C.c_void_p),
                ("parent_material", C.c_void_p)]


class Energy(C.Structure):
    _fields_ = [("exchange", C.c_double), ("anisotropy", C.c_double), ("zeeman", C.c_double),
                ("dmi", C.c_double), ("demag", C.c_double)]

    def total(self):
        return self.exchange + self.anisotropy + self.zeeman + self.dmi + self.demag


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        vp = C.c_void_p
        L.orc_solver_create.restype = vp
        L.orc_solver_create.argtypes = [C.POINTER(Grid), C.POINTER(Material), vp]
        L.orc_solver_destroy.argtypes = [vp]
        L.orc_solver_invalidate.argtypes = [vp]
        L.orc_build_h_eff.argtypes = [vp, dp, dp, C.c_int, dp]
        L.orc_demag_field.argtypes = [vp, dp, dp]
        step_args = [vp, dp, C.POINTER(Params), C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                     dp, C.POINTER(C.c_int), dp]
        L.orc_step_rk45.argtypes = step_args
        L.orc_step_rk23_relax.argtypes = step_args
        L.orc_relax.argtypes = [vp, dp, C.POINTER(Params), C.c_int, C.POINTER(RelaxSettings),
                                C.POINTER(RelaxReport)]
        L.orc_default_relax_settings.argtypes = [C.POINTER(RelaxSettings)]
        L.orc_minimize.argtypes = [vp, dp, C.POINTER(Params), C.c_int, C.POINTER(MinimizeSettings),
                                   C.POINTER(MinimizeReport)]
        L.orc_default_minimize_settings.argtypes = [C.POINTER(MinimizeSettings)]
        L.orc_validated_ratio.restype = C.c_int64
        L.orc_validated_ratio.argtypes = [C.c_int64, C.c_int64, C.c_int64]
        L.orc_sample_bilinear.argtypes = [C.POINTER(Grid), dp, C.c_double, C.c_double, dp]
        L.orc_restrict_m_to_coarse.argtypes = [C.POINTER(Grid), dp, C.c_int32, C.POINTER(AmrPatch), dp]
        L.orc_restrict_l0_to_demag_grid.argtypes = [C.c_int64, dp, C.c_int64, C.c_int64, C.c_int64, dp]
        L.orc_coarse_fft_demag.argtypes = [C.POINTER(Grid), C.POINTER(Material), dp, C.c_int32,
                                           C.POINTER(AmrPatch), C.c_int64, dp, dp]
        L.orc_allfft_demag.argtypes = [C.POINTER(Grid), C.POINTER(Material), dp, vp, C.POINTER(Grid), dp, dp]
        L.orc_energy_breakdown.argtypes = [vp, dp, dp, C.POINTER(Energy)]
        L.orc_torque_metric.restype = C.c_double
        L.orc_torque_metric.argtypes = [C.c_int64, dp, dp, C.c_int]
        L.orc_kernel_components.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int64, C.c_int64,
                                            C.c_double, dp]
        L.orc_demag_kernel_kspace.argtypes = [vp, dp]
        L.orc_demag_kernel_realspace.argtypes = [C.POINTER(Grid), C.c_int64, C.c_int64, dp]
        L.orc_demag_field_direct.argtypes = [C.POINTER(Grid), C.c_double, dp, dp]
        L.orc_demag_field_pbc.argtypes = [C.POINTER(Grid), C.c_double, C.c_int64, C.c_int64, dp, dp]
        L.orc_demag_kernel_kspace_pbc.argtypes = [C.POINTER(Grid), C.c_int64, C.c_int64, dp]
        L.orc_write_llgdmag.argtypes = [C.POINTER(Grid), C.c_int64, C.c_int64, C.c_char_p]
        L.orc_write_llgdmag.restype = C.c_int
        L.orc_demag_field_direct_pbc.argtypes = [C.POINTER(Grid), C.c_double, C.c_int64, C.c_int64, dp, dp]
        L.orc_fft.argtypes = [C.c_int64, dp, C.c_int]
        L.orc_xorshift_f64.argtypes = [C.c_uint64, C.c_int64, dp]
        L.orc_init_random.argtypes = [C.c_int64, C.c_uint64, dp]
        L.orc_init_uniform_with_noise.argtypes = [C.c_int64, dp, C.c_double, C.c_uint64, dp]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
        L.orc_set_parallel_local.argtypes = [C.c_int]
        L.orc_get_parallel_local.restype = C.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _vec3(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(3))


def set_threads(n):
    lib().orc_set_threads(int(n))


def get_threads():
    return lib().orc_get_threads()


def set_parallel_local(on):
    """Also parallelise the per-cell local-term, torque and RK-combination loops
    (the reference runs them serially); results are identical either way."""
    lib().orc_set_parallel_local(1 if on else 0)


def get_parallel_local():
    return bool(lib().orc_get_parallel_local())


def make_grid(nx, ny, dx, dy, dz):
    return Grid(int(nx), int(ny), float(dx), float(dy), float(dz))


def make_material(ms, a_ex, k_u=0.0, easy_axis=(0.0, 0.0, 1.0), dmi=None, demag=False):
    ea = (C.c_double * 3)(*[float(x) for x in easy_axis])
    return Material(float(ms), float(a_ex), float(k_u), ea, float(dmi or 0.0), 0 if dmi is None else 1,
                    1 if demag else 0)


def make_params(gamma, alpha, dt, b_ext=(0.0, 0.0, 0.0)):
    return Params(float(gamma), float(alpha), float(dt), (C.c_double * 3)(*[float(x) for x in b_ext]))


def default_relax_settings(**kw):
    s = RelaxSettings()
    lib().orc_default_relax_settings(C.byref(s))
    for k, v in kw.items():
        if k == "torque_threshold":
            if v is None:
                s.has_torque_threshold = 0
            else:
                s.has_torque_threshold = 1
                s.torque_threshold = float(v)
        else:
            setattr(s, k, v)
    return s


def default_minimize_settings(**kw):
    """MinimizeSettings::default() (minimize.rs:65-92) with keyword overrides; the
    Option fields dm_stop / dm_torque_gate / dm_torque_gate_max take None."""
    s = MinimizeSettings()
    lib().orc_default_minimize_settings(C.byref(s))
    for k, v in kw.items():
        if k in ("dm_stop", "dm_torque_gate", "dm_torque_gate_max"):
            setattr(s, "has_" + k, 0 if v is None else 1)
            setattr(s, k, 0.0 if v is None else float(v))
        else:
            setattr(s, k, v)
    return s


# ---------------------------------------------------------------- AMR demag consumers

def _patches(patches):
    """patches: objects with i0, j0, cnx, cny, ratio, ghost, m ([pny*pnx, 3] float64),
    geom_mask_fine / parent_material (uint8 arrays or None)."""
    arr = (AmrPatch * max(len(patches), 1))()
    keep = []
    for q, p in enumerate(patches):
        m = np.ascontiguousarray(p.m, dtype=np.float64)
        gm = None if p.geom_mask_fine is None else np.ascontiguousarray(p.geom_mask_fine, dtype=np.uint8)
        pm = None if p.parent_material is None else np.ascontiguousarray(p.parent_material, dtype=np.uint8)
        keep += [m, gm, pm]
        arr[q] = AmrPatch(p.i0, p.j0, p.cnx, p.cny, p.ratio, p.ghost, m.ctypes.data,
                          None if gm is None else gm.ctypes.data, None if pm is None else pm.ctypes.data)
    return arr, keep


def validated_ratio(nx, ny, ratio):
    return int(lib().orc_validated_ratio(int(nx), int(ny), int(ratio)))


def sample_bilinear(grid, field, x, y):
    f = np.ascontiguousarray(field, dtype=np.float64)
    out = np.empty(3)
    lib().orc_sample_bilinear(C.byref(grid), _dp(f), float(x), float(y), _dp(out))
    return out


def restrict_m_to_coarse(base, m_coarse, patches):
    mc = np.ascontiguousarray(m_coarse, dtype=np.float64)
    out = np.empty((base.nx * base.ny, 3))
    arr, keep = _patches(patches)
    lib().orc_restrict_m_to_coarse(C.byref(base), _dp(mc), len(patches), arr, _dp(out))
    return out


def restrict_l0_to_demag_grid(nx_l0, l0_m, dnx, dny, ratio):
    m = np.ascontiguousarray(l0_m, dtype=np.float64)
    out = np.empty((dnx * dny, 3))
    lib().orc_restrict_l0_to_demag_grid(int(nx_l0), _dp(m), int(dnx), int(dny), int(ratio), _dp(out))
    return out


def coarse_fft_demag(base, material, m_coarse, patches, ratio=1):
    """compute_coarse_fft_demag (coarse_fft_demag.rs:367-511) with an explicit ratio:
    (b_coarse, [b_patch per patch]) — no patch fields without Material::demag."""
    mc = np.ascontiguousarray(m_coarse, dtype=np.float64)
    bc = np.empty((base.nx * base.ny, 3))
    cells = [(p.cny * p.ratio + 2 * p.ghost) * (p.cnx * p.ratio + 2 * p.ghost) for p in patches]
    bp = np.zeros((max(sum(cells), 1), 3))
    arr, keep = _patches(patches)
    lib().orc_coarse_fft_demag(C.byref(base), C.byref(material), _dp(mc), len(patches), arr, int(ratio), _dp(bc),
                               _dp(bp))
    if not material.demag:
        return bc, []
    out, o = [], 0
    for c in cells:
        out.append(bp[o:o + c].copy())
        o += c
    return bc, out


def allfft_demag(fine, material, m_fine, fine_mask, base):
    m = np.ascontiguousarray(m_fine, dtype=np.float64)
    bf = np.empty((fine.nx * fine.ny, 3))
    bc = np.empty((base.nx * base.ny, 3))
    mk = None if fine_mask is None else np.ascontiguousarray(np.asarray(fine_mask, dtype=np.uint8).reshape(-1))
    lib().orc_allfft_demag(C.byref(fine), C.byref(material), _dp(m), None if mk is None else mk.ctypes.data,
                           C.byref(base), _dp(bf), _dp(bc))
    return bf, bc


class Solver:
    """Oracle solver for one film: grid, material, optional geometry mask."""

    def __init__(self, grid, material, geom_mask=None):
        self.grid = grid
        self.material = material
        self.n = grid.nx * grid.ny
        self._mask = None
        mp = None
        if geom_mask is not None:
            self._mask = np.ascontiguousarray(np.asarray(geom_mask, dtype=np.uint8).reshape(self.n))
            mp = self._mask.ctypes.data_as(C.c_void_p)
        self.h = lib().orc_solver_create(C.byref(grid), C.byref(material), mp)

    def close(self):
        if self.h:
            lib().orc_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def invalidate(self):
        lib().orc_solver_invalidate(self.h)

    def _m(self, m):
        m = np.ascontiguousarray(m, dtype=np.float64)
        assert m.size == self.n * 3
        return m

    def build_h_eff(self, m, b_ext, field_mask=FIELD_FULL):
        m = self._m(m)
        out = np.empty((self.n, 3))
        be = _vec3(b_ext)
        lib().orc_build_h_eff(self.h, _dp(m), _dp(be), int(field_mask), _dp(out))
        return out

    def demag_field(self, m):
        m = self._m(m)
        out = np.empty((self.n, 3))
        lib().orc_demag_field(self.h, _dp(m), _dp(out))
        return out

    def _step(self, fn, m, params, field_mask, max_err, headroom, dt_min, dt_max):
        eps = C.c_double()
        acc = C.c_int()
        dtu = C.c_double()
        fn(self.h, _dp(m), C.byref(params), int(field_mask), float(max_err), float(headroom), float(dt_min),
           float(dt_max), C.byref(eps), C.byref(acc), C.byref(dtu))
        return eps.value, bool(acc.value), dtu.value

    def step_rk45(self, m, params, field_mask, max_err, headroom, dt_min, dt_max):
        """In-place on m (float64 contiguous [n,3]); params.dt updated."""
        assert m.dtype == np.float64 and m.flags.c_contiguous
        return self._step(lib().orc_step_rk45, m, params, field_mask, max_err, headroom, dt_min, dt_max)

    def step_rk23_relax(self, m, params, field_mask, max_err, headroom, dt_min, dt_max):
        assert m.dtype == np.float64 and m.flags.c_contiguous
        return self._step(lib().orc_step_rk23_relax, m, params, field_mask, max_err, headroom, dt_min, dt_max)

    def relax(self, m, params, field_mask, settings):
        assert m.dtype == np.float64 and m.flags.c_contiguous
        rep = RelaxReport()
        lib().orc_relax(self.h, _dp(m), C.byref(params), int(field_mask), C.byref(settings), C.byref(rep))
        return rep

    def minimize(self, m, params, field_mask, settings):
        """minimize_damping_only (minimize.rs:107), in place on m (float64 [n,3])."""
        assert m.dtype == np.float64 and m.flags.c_contiguous
        rep = MinimizeReport()
        lib().orc_minimize(self.h, _dp(m), C.byref(params), int(field_mask), C.byref(settings), C.byref(rep))
        return rep

    def energy(self, m, b_ext):
        m = self._m(m)
        e = Energy()
        be = _vec3(b_ext)
        lib().orc_energy_breakdown(self.h, _dp(m), _dp(be), C.byref(e))
        return e

    def kernel_kspace(self):
        px, py = 2 * self.grid.nx, 2 * self.grid.ny
        out = np.empty(4 * px * py * 2)
        lib().orc_demag_kernel_kspace(self.h, _dp(out))
        return out.view(np.complex128).reshape(4, py, px)


def torque_metric(m, b, metric=TORQUE_MAX):
    m = np.ascontiguousarray(m, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return lib().orc_torque_metric(m.size // 3, _dp(m), _dp(b), int(metric))


def kernel_components(dx, dy, dz, sx, sy, accuracy=10.0):
    out = np.empty(4)
    lib().orc_kernel_components(float(dx), float(dy), float(dz), int(sx), int(sy), float(accuracy), _dp(out))
    return out


def kernel_realspace(grid, pbc_x=0, pbc_y=0):
    px = grid.nx if pbc_x > 0 else 2 * grid.nx
    py = grid.ny if pbc_y > 0 else 2 * grid.ny
    out = np.empty(4 * px * py)
    lib().orc_demag_kernel_realspace(C.byref(grid), int(pbc_x), int(pbc_y), _dp(out))
    return out.reshape(4, py, px)


def demag_field_direct(grid, ms, m):
    m = np.ascontiguousarray(m, dtype=np.float64)
    out = np.empty((grid.nx * grid.ny, 3))
    lib().orc_demag_field_direct(C.byref(grid), float(ms), _dp(m), _dp(out))
    return out


def pad_sizes(grid, pbc_x, pbc_y):
    """Padded FFT sizes of Demag2D::new (demag_fft_uniform.rs:477-478)."""
    return (grid.nx if pbc_x > 0 else 2 * grid.nx), (grid.ny if pbc_y > 0 else 2 * grid.ny)


def demag_field_pbc(grid, ms, pbc_x, pbc_y, m):
    m = np.ascontiguousarray(m, dtype=np.float64)
    out = np.empty((grid.nx * grid.ny, 3))
    lib().orc_demag_field_pbc(C.byref(grid), float(ms), int(pbc_x), int(pbc_y), _dp(m), _dp(out))
    return out


def kernel_kspace_pbc(grid, pbc_x, pbc_y):
    """Unscaled k-space kernel planes [4, py, px] complex (xx, xy, yy, zz)."""
    px, py = pad_sizes(grid, pbc_x, pbc_y)
    out = np.empty(4 * px * py * 2)
    lib().orc_demag_kernel_kspace_pbc(C.byref(grid), int(pbc_x), int(pbc_y), _dp(out))
    return out.view(np.complex128).reshape(4, py, px)


def write_llgdmag(grid, pbc_x, pbc_y, path):
    rc = lib().orc_write_llgdmag(C.byref(grid), int(pbc_x), int(pbc_y), str(path).encode())
    if rc != 0:
        raise OSError(f"cannot write {path}")


def demag_field_direct_pbc(grid, ms, pbc_x, pbc_y, m):
    m = np.ascontiguousarray(m, dtype=np.float64)
    out = np.empty((grid.nx * grid.ny, 3))
    lib().orc_demag_field_direct_pbc(C.byref(grid), float(ms), int(pbc_x), int(pbc_y), _dp(m), _dp(out))
    return out


def fft(x, inverse=False):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128)).copy()
    lib().orc_fft(a.size, a.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)), 1 if inverse else 0)
    return a


def xorshift_f64(seed, count):
    out = np.empty(int(count))
    lib().orc_xorshift_f64(C.c_uint64(seed), int(count), _dp(out))
    return out


def init_random(n, seed):
    out = np.empty((int(n), 3))
    lib().orc_init_random(int(n), C.c_uint64(seed), _dp(out))
    return out


def init_uniform_with_noise(n, direction, noise, seed, m=None):
    out = np.ones((int(n), 3)) if m is None else np.ascontiguousarray(m, dtype=np.float64).copy()
    d = _vec3(direction)
    lib().orc_init_uniform_with_noise(int(n), _dp(d), float(noise), C.c_uint64(seed), _dp(out))
    return out
