"""Python host mirror of llg-sim's uniform-grid API over the C ABI of libllg_b200.so.

The names follow the reference's Rust API (Grid2D, Material, LLGParams,
FieldMask, RelaxSettings, build_h_eff_masked, step_llg_rk45_..._adaptive,
step_llg_rk23_..._relax_adaptive, relax_with_report, compute_energy) so that
code written against the reference reads the same.  Every call goes through
the C ABI declared in include/llg_b200.h; there is no CPU fallback: loading
fails loudly when the CUDA library has not been built.

Arrays are numpy float64 in the reference layout: AoS ``[nx*ny, 3]`` with cell
index ``j*nx + i`` (grid.rs:27-30, vector_field.rs:24-27).
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libllg_b200.so")

# FieldMask (effective_field/mod.rs:38-45)
EXCH_ANIS, EXCH_ANIS_DMI, FULL = 0, 1, 2
# TorqueMetric (relax.rs:32-37)
TORQUE_MAX, TORQUE_MEAN, TORQUE_RMS, TORQUE_MEANSQ = 0, 1, 2, 3
FP32, FP64 = 0, 1
OVF_TEXT, OVF_BINARY4 = 0, 1              # write_ovf2_rectangular_text / _binary4 (ovf.rs:54,153)
MU0 = 4.0 * np.pi * 1e-7                  # params.rs:15
GAMMA_E_RAD_PER_S_T = 1.76085963023e11     # params.rs:16

ERRORS = {-1: "LLG_ERR_INVALID", -2: "LLG_ERR_CUDA", -3: "LLG_ERR_TIMEOUT", -4: "LLG_ERR_NONFINITE",
          -5: "LLG_ERR_OOM", -6: "LLG_ERR_NO_DEVICE"}


class LLGError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class _Grid(C.Structure):
    _fields_ = [("nx", C.c_int64), ("ny", C.c_int64), ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double)]


class _Material(C.Structure):
    _fields_ = [("ms", C.c_double), ("a_ex", C.c_double), ("k_u", C.c_double), ("easy_axis", C.c_double * 3),
                ("dmi", C.c_double), ("has_dmi", C.c_int32), ("demag", C.c_int32)]


class _Params(C.Structure):
    _fields_ = [("gamma", C.c_double), ("alpha", C.c_double), ("dt", C.c_double), ("b_ext", C.c_double * 3)]


class RelaxSettings(C.Structure):
    """RelaxSettings (relax.rs:73-105); defaults from impl Default (relax.rs:107-141)."""
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

    @classmethod
    def default(cls, **kw):
        s = cls()
        lib().llg_default_relax_settings(C.byref(s))
        for k, v in kw.items():
            if k == "torque_threshold":
                s.has_torque_threshold = 0 if v is None else 1
                s.torque_threshold = 0.0 if v is None else float(v)
            else:
                setattr(s, k, v)
        return s

    def copy(self):
        c = RelaxSettings()
        C.memmove(C.byref(c), C.byref(self), C.sizeof(self))
        return c


class RelaxReport(C.Structure):
    _fields_ = [("accepted_steps", C.c_int64), ("rejected_steps", C.c_int64), ("torque_checks", C.c_int64),
                ("torque_field_rebuilds", C.c_int64), ("stop_reason", C.c_int32), ("last_stage_stop", C.c_int32),
                ("has_final_torque", C.c_int32), ("has_final_torque_max", C.c_int32),
                ("final_torque", C.c_double), ("final_torque_max", C.c_double),
                ("final_max_err", C.c_double), ("final_dt", C.c_double)]


class MinimizeSettings(C.Structure):
    """MinimizeSettings (minimize.rs:20-63); defaults from impl Default (minimize.rs:65-92).
    The Option fields dm_stop / dm_torque_gate / dm_torque_gate_max take None in default()."""
    _fields_ = [("torque_threshold", C.c_double), ("max_iters", C.c_int64), ("lambda0", C.c_double),
                ("lambda_min", C.c_double), ("lambda_max", C.c_double), ("grow", C.c_double), ("shrink", C.c_double),
                ("stall_iters", C.c_int64), ("stall_rel", C.c_double), ("min_iters_before_stall", C.c_int64),
                ("has_dm_stop", C.c_int32), ("has_dm_torque_gate", C.c_int32),
                ("has_dm_torque_gate_max", C.c_int32), ("reserved", C.c_int32), ("dm_stop", C.c_double),
                ("dm_samples", C.c_int64), ("dm_torque_gate", C.c_double), ("dm_torque_gate_max", C.c_double),
                ("dm_min_iters", C.c_int64)]

    @classmethod
    def default(cls, **kw):
        s = cls()
        lib().llg_default_minimize_settings(C.byref(s))
        for k, v in kw.items():
            if k in ("dm_stop", "dm_torque_gate", "dm_torque_gate_max"):
                setattr(s, "has_" + k, 0 if v is None else 1)
                setattr(s, k, 0.0 if v is None else float(v))
            else:
                setattr(s, k, v)
        return s

    def copy(self):
        c = MinimizeSettings()
        C.memmove(C.byref(c), C.byref(self), C.sizeof(self))
        return c


class MinimizeReport(C.Structure):
    """MinimizeReport (minimize.rs:94-104)."""
    _fields_ = [("iters", C.c_int64), ("converged", C.c_int32), ("stalled", C.c_int32),
                ("dm_converged", C.c_int32), ("reserved", C.c_int32), ("final_torque", C.c_double),
                ("final_max_dm", C.c_double), ("final_tmean", C.c_double), ("final_lambda", C.c_double)]


class _AmrPatch(C.Structure):
    _fields_ = [("i0", C.c_int64), ("j0", C.c_int64), ("cnx", C.c_int64), ("cny", C.c_int64),
                ("ratio", C.c_int64), ("ghost", C.c_int64), ("m", C.c_void_p), ("geom_mask_fine", C.c_void_p),
                ("parent_material", C.c_void_p)]


class _OvfMeta(C.Structure):
    _fields_ = [("title", C.c_char_p), ("desc_lines", C.POINTER(C.c_char_p)), ("n_desc", C.c_int32),
                ("valuelabels", C.c_char_p * 3), ("valueunits", C.c_char_p * 3)]


class EnergyBreakdown(C.Structure):
    _fields_ = [("exchange", C.c_double), ("anisotropy", C.c_double), ("zeeman", C.c_double),
                ("dmi", C.c_double), ("demag", C.c_double)]

    def total(self):
        return self.exchange + self.anisotropy + self.zeeman + self.dmi + self.demag


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    """The loaded C ABI.  Raises if the CUDA library is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `make -C {_HERE}` (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        vp, dp, i32, i64 = C.c_void_p, C.POINTER(C.c_double), C.c_int32, C.c_int64
        P = C.POINTER
        sig = {
            "llg_abi_version": (C.c_int, []),
            "llg_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
            "llg_ctx_create": (C.c_int, [C.c_int, P(vp)]),
            "llg_ctx_destroy": (C.c_int, [vp]),
            "llg_solver_create": (C.c_int, [vp, P(_Grid), P(_Material), i32, vp, P(vp)]),
            "llg_solver_destroy": (C.c_int, [vp]),
            "llg_solver_set_stream": (C.c_int, [vp, vp]),
            "llg_solver_sync": (C.c_int, [vp]),
            "llg_set_state": (C.c_int, [vp, dp]),
            "llg_get_state": (C.c_int, [vp, dp]),
            "llg_mean_m": (C.c_int, [vp, dp]),
            "llg_build_h_eff": (C.c_int, [vp, P(_Params), i32, dp]),
            "llg_compute_demag_field": (C.c_int, [vp, dp]),
            "llg_step_rk45": (C.c_int, [vp, P(_Params), i32, C.c_double, C.c_double, C.c_double, C.c_double,
                                        dp, P(i32), dp]),
            "llg_step_rk23_relax": (C.c_int, [vp, P(_Params), i32, C.c_double, C.c_double, C.c_double,
                                              C.c_double, dp, P(i32), dp]),
            "llg_run_rk45": (C.c_int, [vp, P(_Params), i32, C.c_double, C.c_double, C.c_double, C.c_double,
                                       i64, C.c_double, i64, P(i64), P(i64), dp]),
            "llg_relax": (C.c_int, [vp, P(_Params), i32, P(RelaxSettings), P(RelaxReport)]),
            "llg_default_relax_settings": (None, [P(RelaxSettings)]),
            "llg_minimize": (C.c_int, [vp, P(_Params), i32, P(MinimizeSettings), P(MinimizeReport)]),
            "llg_default_minimize_settings": (None, [P(MinimizeSettings)]),
            "llg_batch_minimize": (C.c_int, [vp, P(_Params), i32, P(MinimizeSettings), P(MinimizeReport)]),
            "llg_compute_energy": (C.c_int, [vp, dp, P(EnergyBreakdown)]),
            "llg_torque_metric": (C.c_int, [vp, P(_Params), i32, i32, dp]),
            "llg_demag_kernel_kspace": (C.c_int, [vp, dp]),
            "llg_profile_stage": (C.c_int, [vp, P(_Params), i32, i32, dp]),
            "llg_solver_launch_count": (C.c_int, [vp, P(i64)]),
            "llg_solver_fft_plans": (C.c_int, [vp, P(i32), P(i32)]),
            "llg_batch_fft_plans": (C.c_int, [vp, P(i32), i32, P(i32), i32]),
            "llg_demag_field_noalloc": (C.c_int, [i64, i64, C.c_double, vp, vp, vp, vp]),
            "llg_batch_create": (C.c_int, [vp, i32, P(_Grid), P(_Material), i32, P(C.c_void_p), P(vp)]),
            "llg_batch_destroy": (C.c_int, [vp]),
            "llg_batch_set_stream": (C.c_int, [vp, vp]),
            "llg_batch_set_state": (C.c_int, [vp, i32, dp]),
            "llg_batch_get_state": (C.c_int, [vp, i32, dp]),
            "llg_batch_mean_m": (C.c_int, [vp, dp]),
            "llg_batch_step_rk45": (C.c_int, [vp, P(_Params), i32, C.c_double, C.c_double, C.c_double, C.c_double,
                                              dp, P(i32), dp]),
            "llg_batch_run_rk45": (C.c_int, [vp, P(_Params), i32, C.c_double, C.c_double, C.c_double, C.c_double,
                                             i64, C.c_double, i64, P(i64), P(i64), dp]),
            "llg_batch_relax": (C.c_int, [vp, P(_Params), i32, P(RelaxSettings), P(RelaxReport)]),
            "llg_batch_compute_energy": (C.c_int, [vp, dp, P(EnergyBreakdown)]),
            "llg_batch_launch_count": (C.c_int, [vp, P(i64)]),
            "llg_demag_op_create": (C.c_int, [vp, P(_Grid), i64, i64, C.c_char_p, P(i32), P(vp)]),
            "llg_demag_op_destroy": (C.c_int, [vp]),
            "llg_demag_op_field": (C.c_int, [vp, C.c_double, dp, dp]),
            "llg_demag_op_kspace": (C.c_int, [vp, dp]),
            "llg_demag_op_save": (C.c_int, [vp, C.c_char_p]),
            "llg_demag_cache_filename": (C.c_int, [P(_Grid), i64, i64, C.c_char_p, i64]),
            "llg_ovf2_write": (C.c_int, [C.c_char_p, P(_Grid), dp, P(_OvfMeta), i32]),
            "llg_ovf2_write_state": (C.c_int, [vp, C.c_char_p, P(_OvfMeta), i32]),
            "llg_batch_ovf2_write_state": (C.c_int, [vp, i32, C.c_char_p, P(_OvfMeta), i32]),
            "llg_ovf_format_exp": (C.c_int, [C.c_double, i32, C.c_char_p, i64]),
            "llg_amr_validated_ratio": (i64, [i64, i64, i64]),
            "llg_amr_patch_cells": (i64, [P(_AmrPatch)]),
            "llg_amr_demag_create": (C.c_int, [vp, P(_Grid), i64, P(vp)]),
            "llg_amr_demag_ratio": (C.c_int, [vp, P(i64)]),
            "llg_amr_demag_destroy": (C.c_int, [vp]),
            "llg_amr_restrict_m": (C.c_int, [vp, dp, i32, P(_AmrPatch), dp]),
            "llg_coarse_fft_demag": (C.c_int, [vp, P(_Material), dp, i32, P(_AmrPatch), dp, dp]),
            "llg_amr_allfft_demag": (C.c_int, [vp, P(_Material), dp, vp, P(_Grid), dp, dp]),
            "llg_amr_allfft_demag_device": (C.c_int, [vp, P(_Material), vp, vp, P(_Grid), vp, vp, vp]),
            "llg_warmstart_param_count": (i64, []),
            "llg_warmstart_create": (C.c_int, [vp, P(C.c_float), i64, P(vp)]),
            "llg_warmstart_destroy": (C.c_int, [vp]),
            "llg_warmstart_forward": (C.c_int, [vp, i64, i64, i64, dp, vp, dp, dp]),
            "llg_batch_warm_start": (C.c_int, [vp, vp, dp]),
            "llg_warmstart_set_spin_limit": (C.c_int, [vp, i64]),
            "llg_wstrain_create": (C.c_int, [vp, P(C.c_float), i64, i64, P(vp)]),
            "llg_wstrain_destroy": (C.c_int, [vp]),
            "llg_wstrain_set_spin_limit": (C.c_int, [vp, i64]),
            "llg_wstrain_gradients": (C.c_int, [vp, i64, i64, i64, vp, vp, vp, vp, dp, P(C.c_float)]),
            "llg_wstrain_step": (C.c_int, [vp, i64, i64, i64, vp, vp, vp, vp, C.c_float, C.c_float, C.c_float,
                                           C.c_float, dp]),
            "llg_wstrain_sync": (C.c_int, [vp]),
            "llg_wstrain_get_params": (C.c_int, [vp, P(C.c_float)]),
            "llg_init_random": (None, [i64, C.c_uint64, dp]),
            "llg_init_uniform_with_noise": (None, [i64, dp, C.c_double, C.c_uint64, dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def declared_symbols(header=None):
    """Function names declared by the C ABI header include/llg_b200.h."""
    import re
    header = header or os.path.join(_HERE, "..", "include", "llg_b200.h")
    src = re.sub(r"/\*.*?\*/", "", open(header).read(), flags=re.S)
    return sorted(set(re.findall(r"\b(llg_[a-z0-9_]+)\s*\(", src)))


def last_error():
    buf = C.create_string_buffer(1024)
    lib().llg_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def _check(rc):
    if rc != 0:
        raise LLGError(rc, last_error())


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Grid2D:
    """Grid2D (grid.rs:4-31)."""

    def __init__(self, nx, ny, dx, dy, dz):
        self.nx, self.ny, self.dx, self.dy, self.dz = int(nx), int(ny), float(dx), float(dy), float(dz)

    def n_cells(self):
        return self.nx * self.ny

    def cell_volume(self):
        return self.dx * self.dy * self.dz

    def _c(self):
        return _Grid(self.nx, self.ny, self.dx, self.dy, self.dz)


class Material:
    """Material (params.rs:170-184); dmi=None means DMI off."""

    def __init__(self, ms, a_ex, k_u=0.0, easy_axis=(0.0, 0.0, 1.0), dmi=None, demag=False):
        self.ms, self.a_ex, self.k_u = float(ms), float(a_ex), float(k_u)
        self.easy_axis = tuple(float(x) for x in easy_axis)
        self.dmi = None if dmi is None else float(dmi)
        self.demag = bool(demag)

    def _c(self):
        return _Material(self.ms, self.a_ex, self.k_u, (C.c_double * 3)(*self.easy_axis),
                         0.0 if self.dmi is None else self.dmi, 0 if self.dmi is None else 1, 1 if self.demag else 0)


class LLGParams:
    """LLGParams (params.rs:213-219); dt is mutated by the steppers as in the reference."""

    def __init__(self, gamma, alpha, dt, b_ext=(0.0, 0.0, 0.0)):
        self.gamma, self.alpha, self.dt = float(gamma), float(alpha), float(dt)
        self.b_ext = tuple(float(x) for x in b_ext)

    def _c(self):
        return _Params(self.gamma, self.alpha, self.dt, (C.c_double * 3)(*self.b_ext))


_ctx_cache = {}


def _ctx(device):
    if device not in _ctx_cache:
        h = C.c_void_p()
        _check(lib().llg_ctx_create(int(device), C.byref(h)))
        _ctx_cache[device] = h
    return _ctx_cache[device]


class Solver:
    """One film on one GPU: grid + material (+ optional geometry mask), resident m."""

    def __init__(self, grid, material, precision=FP32, geom_mask=None, device=0):
        self.grid, self.material, self.precision = grid, material, precision
        self.n = grid.n_cells()
        mp = None
        if geom_mask is not None:
            self._mask = np.ascontiguousarray(np.asarray(geom_mask).reshape(self.n).astype(np.uint8))
            mp = self._mask.ctypes.data_as(C.c_void_p)
        h = C.c_void_p()
        g, m = grid._c(), material._c()
        _check(lib().llg_solver_create(_ctx(device), C.byref(g), C.byref(m), int(precision), mp, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().llg_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        _check(lib().llg_solver_set_stream(self.h, C.c_void_p(stream_ptr)))

    def sync(self):
        _check(lib().llg_solver_sync(self.h))

    def set_state(self, m):
        m = np.ascontiguousarray(m, dtype=np.float64)
        assert m.size == 3 * self.n
        _check(lib().llg_set_state(self.h, _dp(m)))

    def set_state_ptr(self, host_ptr):
        """Upload from a raw host pointer (e.g. pinned memory) of 3n doubles."""
        _check(lib().llg_set_state(self.h, C.cast(C.c_void_p(host_ptr), C.POINTER(C.c_double))))

    def get_state(self):
        out = np.empty((self.n, 3))
        _check(lib().llg_get_state(self.h, _dp(out)))
        return out

    def get_state_ptr(self, host_ptr):
        _check(lib().llg_get_state(self.h, C.cast(C.c_void_p(host_ptr), C.POINTER(C.c_double))))

    def mean_m(self):
        out = np.empty(3)
        _check(lib().llg_mean_m(self.h, _dp(out)))
        return out

    def build_h_eff(self, params, field_mask=FULL):
        out = np.empty((self.n, 3))
        p = params._c()
        _check(lib().llg_build_h_eff(self.h, C.byref(p), int(field_mask), _dp(out)))
        return out

    def compute_demag_field(self):
        out = np.empty((self.n, 3))
        _check(lib().llg_compute_demag_field(self.h, _dp(out)))
        return out

    def _step(self, fn, params, field_mask, max_err, headroom, dt_min, dt_max):
        p = params._c()
        eps, acc, dtu = C.c_double(), C.c_int32(), C.c_double()
        _check(fn(self.h, C.byref(p), int(field_mask), float(max_err), float(headroom), float(dt_min),
                  float(dt_max), C.byref(eps), C.byref(acc), C.byref(dtu)))
        params.dt = p.dt
        return eps.value, bool(acc.value), dtu.value

    def step_rk45(self, params, field_mask, max_err, headroom, dt_min, dt_max):
        """step_llg_rk45_recompute_field_masked_adaptive (llg.rs:795): (eps, accepted, dt_used)."""
        return self._step(lib().llg_step_rk45, params, field_mask, max_err, headroom, dt_min, dt_max)

    def step_rk23_relax(self, params, field_mask, max_err, headroom, dt_min, dt_max):
        """step_llg_rk23_recompute_field_masked_relax_adaptive (llg.rs:278)."""
        return self._step(lib().llg_step_rk23_relax, params, field_mask, max_err, headroom, dt_min, dt_max)

    def run_rk45(self, params, field_mask, max_err, headroom, dt_min, dt_max, n_accepted=-1,
                 t_end=float("inf"), max_attempts=-1):
        p = params._c()
        a, r, t = C.c_int64(), C.c_int64(), C.c_double()
        _check(lib().llg_run_rk45(self.h, C.byref(p), int(field_mask), float(max_err), float(headroom),
                                  float(dt_min), float(dt_max), int(n_accepted), float(t_end), int(max_attempts),
                                  C.byref(a), C.byref(r), C.byref(t)))
        params.dt = p.dt
        return a.value, r.value, t.value

    def relax(self, params, field_mask, settings):
        """relax_with_report (relax.rs:334); settings.max_err is written back."""
        p = params._c()
        rep = RelaxReport()
        _check(lib().llg_relax(self.h, C.byref(p), int(field_mask), C.byref(settings), C.byref(rep)))
        params.dt = p.dt
        return rep

    def minimize(self, params, field_mask, settings):
        """minimize_damping_only (minimize.rs:107): the resident state is updated in place."""
        p = params._c()
        rep = MinimizeReport()
        _check(lib().llg_minimize(self.h, C.byref(p), int(field_mask), C.byref(settings), C.byref(rep)))
        return rep

    def write_ovf2(self, path, meta, fmt=OVF_BINARY4):
        """OVF 2.0 file of the resident m (write_ovf2_rectangular_binary4 / _text, ovf.rs:54-251)."""
        cm = meta._c()
        _check(lib().llg_ovf2_write_state(self.h, str(path).encode(), C.byref(cm), int(fmt)))

    def compute_energy(self, b_ext):
        be = np.ascontiguousarray(np.asarray(b_ext, dtype=np.float64).reshape(3))
        e = EnergyBreakdown()
        _check(lib().llg_compute_energy(self.h, _dp(be), C.byref(e)))
        return e

    def torque_metric(self, params, field_mask, metric=TORQUE_MAX):
        p = params._c()
        out = C.c_double()
        _check(lib().llg_torque_metric(self.h, C.byref(p), int(field_mask), int(metric), C.byref(out)))
        return out.value

    def profile_stage(self, params, field_mask=FULL, reps=20):
        """Milliseconds per pass of one RK45 stage: row forward, column, row inverse,
        fused row pass (ending the stage and starting the next; 0 if unused)."""
        p = params._c()
        out = np.empty(4)
        _check(lib().llg_profile_stage(self.h, C.byref(p), int(field_mask), int(reps), _dp(out)))
        return out

    def fft_plans(self):
        """(row plan, column form) the autotuner chose: row plan 0 default / 1 alternative; column form
        2 * plan + lean (lean: tables and kernel columns read through L1); -1 generic kernels."""
        r, c = C.c_int32(), C.c_int32()
        _check(lib().llg_solver_fft_plans(self.h, C.byref(r), C.byref(c)))
        return r.value, c.value

    def launch_count(self):
        out = C.c_int64()
        _check(lib().llg_solver_launch_count(self.h, C.byref(out)))
        return out.value

    def kernel_kspace(self):
        """Real Fourier planes (xx, xy, yy, zz) of K on ky in [0,ny], kx in [0,nx]: shape [4, ny+1, nx+1]."""
        out = np.empty(4 * (self.grid.nx + 1) * (self.grid.ny + 1))
        _check(lib().llg_demag_kernel_kspace(self.h, _dp(out)))
        return out.reshape(4, self.grid.ny + 1, self.grid.nx + 1)


class Batch:
    """Independent films of possibly different sizes advanced together: one launch
    per pass over all films, per-film dt and acceptance, device-side relax."""

    def __init__(self, grids, materials, precision=FP32, masks=None, device=0):
        self.n = len(grids)
        self.grids, self.materials, self.precision = list(grids), list(materials), precision
        G = (_Grid * self.n)(*[g._c() for g in grids])
        M = (_Material * self.n)(*[m._c() for m in materials])
        self._masks = []
        mp = None
        if masks is not None:
            arr = (C.c_void_p * self.n)()
            for i, mk in enumerate(masks):
                if mk is None:
                    arr[i] = None
                else:
                    a = np.ascontiguousarray(np.asarray(mk).reshape(-1).astype(np.uint8))
                    self._masks.append(a)
                    arr[i] = a.ctypes.data_as(C.c_void_p)
            mp = arr
        h = C.c_void_p()
        _check(lib().llg_batch_create(_ctx(device), self.n, G, M, int(precision), mp, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().llg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        _check(lib().llg_batch_set_stream(self.h, C.c_void_p(stream_ptr)))

    def set_state(self, f, m):
        m = np.ascontiguousarray(m, dtype=np.float64)
        assert m.size == 3 * self.grids[f].n_cells()
        _check(lib().llg_batch_set_state(self.h, int(f), _dp(m)))

    def get_state(self, f):
        out = np.empty((self.grids[f].n_cells(), 3))
        _check(lib().llg_batch_get_state(self.h, int(f), _dp(out)))
        return out

    def mean_m(self):
        out = np.empty((self.n, 3))
        _check(lib().llg_batch_mean_m(self.h, _dp(out)))
        return out

    def _params(self, params):
        assert len(params) == self.n
        return (_Params * self.n)(*[p._c() for p in params])

    def step_rk45(self, params, field_mask, max_err, headroom, dt_min, dt_max):
        P = self._params(params)
        eps, dtu = np.empty(self.n), np.empty(self.n)
        acc = (C.c_int32 * self.n)()
        _check(lib().llg_batch_step_rk45(self.h, P, int(field_mask), float(max_err), float(headroom), float(dt_min),
                                         float(dt_max), _dp(eps), acc, _dp(dtu)))
        for i, p in enumerate(params):
            p.dt = P[i].dt
        return eps, np.array(acc[:], dtype=bool), dtu

    def run_rk45(self, params, field_mask, max_err, headroom, dt_min, dt_max, n_accepted=-1, t_end=float("inf"),
                 max_attempts=-1):
        P = self._params(params)
        a, r = (C.c_int64 * self.n)(), (C.c_int64 * self.n)()
        t = np.empty(self.n)
        _check(lib().llg_batch_run_rk45(self.h, P, int(field_mask), float(max_err), float(headroom), float(dt_min),
                                        float(dt_max), int(n_accepted), float(t_end), int(max_attempts), a, r,
                                        _dp(t)))
        for i, p in enumerate(params):
            p.dt = P[i].dt
        return np.array(a[:]), np.array(r[:]), t

    def relax(self, params, field_mask, settings):
        P = self._params(params)
        reps = (RelaxReport * self.n)()
        _check(lib().llg_batch_relax(self.h, P, int(field_mask), C.byref(settings), reps))
        for i, p in enumerate(params):
            p.dt = P[i].dt
        return list(reps)

    def minimize(self, params, field_mask, settings):
        """minimize_damping_only (minimize.rs:107) for every film; one report per film."""
        P = self._params(params)
        reps = (MinimizeReport * self.n)()
        _check(lib().llg_batch_minimize(self.h, P, int(field_mask), C.byref(settings), reps))
        return list(reps)

    def write_ovf2(self, f, path, meta, fmt=OVF_BINARY4):
        cm = meta._c()
        _check(lib().llg_batch_ovf2_write_state(self.h, int(f), str(path).encode(), C.byref(cm), int(fmt)))

    def warm_start(self, net, b_exts):
        """Replace every film's state by the warm-start network's proposal (on the device)."""
        be = np.ascontiguousarray(np.asarray(b_exts, dtype=np.float64).reshape(self.n, 3))
        _check(lib().llg_batch_warm_start(self.h, net.h, _dp(be)))

    def compute_energy(self, b_exts):
        be = np.ascontiguousarray(np.asarray(b_exts, dtype=np.float64).reshape(self.n, 3))
        out = (EnergyBreakdown * self.n)()
        _check(lib().llg_batch_compute_energy(self.h, _dp(be), out))
        return list(out)

    def launch_count(self):
        out = C.c_int64()
        _check(lib().llg_batch_launch_count(self.h, C.byref(out)))
        return out.value


def demag_field_noalloc(nx, ny, ms, m_dev_ptr, kernel_planes_dev_ptr, b_dev_ptr, stream_ptr=0):
    """Demag field with no device allocation (raw device pointers, see include/llg_b200.h)."""
    _check(lib().llg_demag_field_noalloc(int(nx), int(ny), float(ms), C.c_void_p(m_dev_ptr),
                                         C.c_void_p(kernel_planes_dev_ptr), C.c_void_p(b_dev_ptr),
                                         C.c_void_p(stream_ptr)))


class DemagOp:
    """Demag2D for pbc_x / pbc_y periodic images (0 = open; demag_fft_uniform.rs:434-770),
    FP64.  With `cache_path`, a matching LLGDMAG v2 kernel file is loaded, else the
    kernel is built and written there; `loaded` tells which."""

    def __init__(self, grid, pbc_x=0, pbc_y=0, cache_path=None, device=0):
        self.grid, self.pbc_x, self.pbc_y = grid, int(pbc_x), int(pbc_y)
        self.px = grid.nx if pbc_x > 0 else 2 * grid.nx
        self.py = grid.ny if pbc_y > 0 else 2 * grid.ny
        h = C.c_void_p()
        ld = C.c_int32(0)
        g = grid._c()
        _check(lib().llg_demag_op_create(_ctx(device), C.byref(g), self.pbc_x, self.pbc_y,
                                         None if cache_path is None else str(cache_path).encode(), C.byref(ld),
                                         C.byref(h)))
        self.h, self.loaded = h, bool(ld.value)

    def close(self):
        if getattr(self, "h", None):
            lib().llg_demag_op_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field(self, ms, m):
        """compute_demag_field_pbc (demag.rs:146-156): B_demag [n, 3] of Ms m."""
        m = np.ascontiguousarray(m, dtype=np.float64)
        out = np.empty((self.grid.nx * self.grid.ny, 3))
        _check(lib().llg_demag_op_field(self.h, float(ms), _dp(m), _dp(out)))
        return out

    def kspace(self):
        """Unscaled kernel spectrum [4, py, px] complex (xx, xy, yy, zz)."""
        out = np.empty(4 * self.px * self.py * 2)
        _check(lib().llg_demag_op_kspace(self.h, _dp(out)))
        return out.view(np.complex128).reshape(4, self.py, self.px)

    def save(self, path):
        _check(lib().llg_demag_op_save(self.h, str(path).encode()))


class AmrPatch:
    """Patch2D (amr/patch.rs:15-80) as the demag consumers read it: coarse_rect
    (i0, j0, cnx, cny) in base cells, ratio relative to the base grid, ghost width,
    m on the patch grid incl. ghosts ([pny*pnx, 3]), optional fine geometry mask
    and parent_material flags ([cny*cnx])."""

    def __init__(self, i0, j0, cnx, cny, ratio, ghost, m, geom_mask_fine=None, parent_material=None):
        self.i0, self.j0, self.cnx, self.cny = int(i0), int(j0), int(cnx), int(cny)
        self.ratio, self.ghost = int(ratio), int(ghost)
        self.pnx = self.cnx * self.ratio + 2 * self.ghost
        self.pny = self.cny * self.ratio + 2 * self.ghost
        self.m = np.ascontiguousarray(m, dtype=np.float64).reshape(self.pnx * self.pny, 3)
        self.geom_mask_fine = None if geom_mask_fine is None else \
            np.ascontiguousarray(np.asarray(geom_mask_fine, dtype=np.uint8).reshape(-1))
        self.parent_material = None if parent_material is None else \
            np.ascontiguousarray(np.asarray(parent_material, dtype=np.uint8).reshape(-1))

    def cell_center_xy(self, i, j, base_grid):
        """Patch2D::cell_center_xy (amr/patch.rs:377-387)."""
        dx, dy = base_grid.dx / self.ratio, base_grid.dy / self.ratio
        return ((self.i0 * self.ratio + (i - self.ghost) + 0.5) * dx,
                (self.j0 * self.ratio + (j - self.ghost) + 0.5) * dy)

    def _c(self):
        ptr = lambda a: None if a is None else a.ctypes.data
        return _AmrPatch(self.i0, self.j0, self.cnx, self.cny, self.ratio, self.ghost, self.m.ctypes.data,
                         ptr(self.geom_mask_fine), ptr(self.parent_material))


def _patch_array(patches):
    arr = (_AmrPatch * max(len(patches), 1))()
    for q, p in enumerate(patches):
        arr[q] = p._c()
    return arr


def validated_ratio(nx, ny, ratio):
    """validated_ratio (coarse_fft_demag.rs:118-150)."""
    return int(lib().llg_amr_validated_ratio(int(nx), int(ny), int(ratio)))


def coarsen_ratio_from_env():
    """demag_coarsen_ratio (coarse_fft_demag.rs:82-111): LLG_DEMAG_COARSEN_RATIO, 1 when
    unset, not a positive integer or not a power of two."""
    raw = os.environ.get("LLG_DEMAG_COARSEN_RATIO")
    if raw is None:
        return 1
    try:
        r = int(raw.strip())
    except ValueError:
        return 1
    if r < 1 or (r & (r - 1)) != 0:
        return 1
    return r


class AmrDemag:
    """Coarse-FFT AMR demag (compute_coarse_fft_demag, coarse_fft_demag.rs:367-511) for
    one base grid and coarsening ratio, on the GPU."""

    def __init__(self, base_grid, coarsen_ratio=1, device=0):
        self.base = base_grid
        h = C.c_void_p()
        g = base_grid._c()
        _check(lib().llg_amr_demag_create(_ctx(device), C.byref(g), int(coarsen_ratio), C.byref(h)))
        self.h = h
        r = C.c_int64()
        _check(lib().llg_amr_demag_ratio(self.h, C.byref(r)))
        self.ratio = r.value

    def close(self):
        if getattr(self, "h", None):
            lib().llg_amr_demag_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def restrict_m(self, m_coarse, patches):
        """restrict_m_to_coarse (coarse_fft_demag.rs:170-240): the enhanced L0 m."""
        mc = np.ascontiguousarray(m_coarse, dtype=np.float64)
        out = np.empty((self.base.nx * self.base.ny, 3))
        _check(lib().llg_amr_restrict_m(self.h, _dp(mc), len(patches), _patch_array(patches), _dp(out)))
        return out

    def compute(self, material, m_coarse, patches):
        """Returns (b_coarse [n, 3], [b_patch [pny*pnx, 3] per patch]); without
        Material::demag the patch list is empty, as in the reference."""
        mc = np.ascontiguousarray(m_coarse, dtype=np.float64)
        bc = np.empty((self.base.nx * self.base.ny, 3))
        cells = [p.pnx * p.pny for p in patches]
        bp = np.empty((max(sum(cells), 1), 3))
        mat = material._c()
        _check(lib().llg_coarse_fft_demag(self.h, C.byref(mat), _dp(mc), len(patches), _patch_array(patches),
                                          _dp(bc), _dp(bp)))
        if not material.demag:
            return bc, []
        out, o = [], 0
        for c in cells:
            out.append(bp[o:o + c].copy())
            o += c
        return bc, out


def allfft_demag(fine_op, material, m_fine, fine_mask, base_grid):
    """AllFft branch of AmrStepper::compute_demag (amr/stepper.rs:799-835): returns
    (b_fine [nf, 3], b_coarse [nb, 3]); fine_op is a DemagOp of the fine grid (pbc 0, 0)."""
    m = np.ascontiguousarray(m_fine, dtype=np.float64)
    nf = fine_op.grid.nx * fine_op.grid.ny
    bf = np.empty((nf, 3))
    bc = np.empty((base_grid.nx * base_grid.ny, 3))
    mk = None if fine_mask is None else np.ascontiguousarray(np.asarray(fine_mask, dtype=np.uint8).reshape(-1))
    mat = material._c()
    g = base_grid._c()
    _check(lib().llg_amr_allfft_demag(fine_op.h, C.byref(mat), _dp(m), None if mk is None else mk.ctypes.data,
                                      C.byref(g), _dp(bf), _dp(bc)))
    return bf, bc


def allfft_demag_device(fine_op, material, m_ptr, mask_ptr, base_grid, b_fine_ptr, b_coarse_ptr, stream_ptr=0):
    """AllFft demag on device arrays (integers, e.g. torch tensors' data_ptr()): m_fine and
    b_fine AoS float64 [ny*nx][3] of the fine grid, b_coarse of the base grid, mask uint8 or 0;
    asynchronous on the stream."""
    mc = material._c()
    bg = base_grid._c()
    _check(lib().llg_amr_allfft_demag_device(fine_op.h, C.byref(mc), m_ptr, mask_ptr or None, C.byref(bg),
                                             b_fine_ptr, b_coarse_ptr, stream_ptr or None))


# ------------------------------------------------------------------ OVF 2.0 (ovf.rs)


def rust_exp(v, precision):
    """Rust's `{:.<precision>e}` of v (llg_ovf_format_exp)."""
    buf = C.create_string_buffer(96)
    _check(lib().llg_ovf_format_exp(float(v), int(precision), buf, 96))
    return buf.value.decode()


class OvfMeta:
    """OvfMeta (ovf.rs:17-45)."""

    def __init__(self, title="", desc_lines=None, valuelabels=("", "", ""), valueunits=("", "", "")):
        self.title = title
        self.desc_lines = list(desc_lines or [])
        self.valuelabels = tuple(valuelabels)
        self.valueunits = tuple(valueunits)

    @classmethod
    def magnetization(cls):
        return cls("m", [], ("m_x", "m_y", "m_z"), ("1", "1", "1"))

    def with_total_sim_time(self, t_s):
        """MuMax-style time line (ovf.rs:36-40)."""
        self.desc_lines.append(f"Total simulation time:  {rust_exp(t_s, 16)}  s")
        return self

    def push_desc_line(self, s):
        self.desc_lines.append(str(s))

    def _c(self):
        enc = lambda x: str(x).encode()
        self._keep = (C.c_char_p * max(len(self.desc_lines), 1))(*[enc(d) for d in self.desc_lines])
        return _OvfMeta(enc(self.title), self._keep, len(self.desc_lines),
                        (C.c_char_p * 3)(*[enc(x) for x in self.valuelabels]),
                        (C.c_char_p * 3)(*[enc(x) for x in self.valueunits]))


def write_ovf2_rectangular_text(path, grid, m, meta):
    m = np.ascontiguousarray(m, dtype=np.float64)
    g, cm = grid._c(), meta._c()
    _check(lib().llg_ovf2_write(str(path).encode(), C.byref(g), _dp(m), C.byref(cm), OVF_TEXT))


def write_ovf2_rectangular_binary4(path, grid, m, meta):
    m = np.ascontiguousarray(m, dtype=np.float64)
    g, cm = grid._c(), meta._c()
    _check(lib().llg_ovf2_write(str(path).encode(), C.byref(g), _dp(m), C.byref(cm), OVF_BINARY4))


class OvfSeries:
    """OvfSeries (ovf.rs:255-316): binary4 dumps every `every` seconds of simulated
    time.  `write(path, meta)` writes the current state (e.g. a Solver's
    write_ovf2 with OVF_BINARY4)."""

    def __init__(self, directory, every_s):
        os.makedirs(directory, exist_ok=True)
        self.dir = directory
        self.every = max(float(every_s), 0.0)
        self.next_dump = 0.0
        self.frame = 0

    def dump_initial(self, write, make_path, meta):
        self.next_dump = 0.0
        write(make_path(self.frame, 0.0), meta)
        self.frame += 1
        self.next_dump = self.every

    def maybe_dump_due(self, write, t_approx, make_path, meta_builder):
        if self.every <= 0.0:
            return
        eps = 1e-15
        while t_approx + eps >= self.next_dump:
            t = self.next_dump
            write(make_path(self.frame, t), meta_builder(t))
            self.frame += 1
            self.next_dump += self.every


def demag_cache_filename(grid, pbc_x=0, pbc_y=0):
    """The reference's cache path for this grid (demag_cache_path, demag_fft_uniform.rs:261-277)."""
    buf = C.create_string_buffer(512)
    g = grid._c()
    _check(lib().llg_demag_cache_filename(C.byref(g), int(pbc_x), int(pbc_y), buf, 512))
    return buf.value.decode()


class WarmStartNet:
    """Learned warm start: six 3x3 convolutions (32 channels, BF16 on the tensor
    cores) from (m, inside, B_ext/0.05 T) to a proposal m.  `params` is the flat
    FP32 vector of per-layer W[cout][3][3][cin] then b[cout]."""

    LAYERS = ((7, 32), (32, 32), (32, 32), (32, 32), (32, 32), (32, 3))

    @staticmethod
    def param_count():
        return int(lib().llg_warmstart_param_count())

    def __init__(self, params, device=0):
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float32).reshape(-1))
        h = C.c_void_p()
        _check(lib().llg_warmstart_create(_ctx(device), p.ctypes.data_as(C.POINTER(C.c_float)), p.size,
                                          C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().llg_warmstart_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_spin_limit(self, polls):
        """Bound (in polls) of the network's tensor-core waits."""
        _check(lib().llg_warmstart_set_spin_limit(self.h, int(polls)))

    def forward(self, m, mask, b_ext, ny, nx):
        """m [nimg, ny*nx, 3] (or one image), mask [nimg, ny*nx] or None, b_ext [nimg, 3]."""
        m = np.ascontiguousarray(np.asarray(m, dtype=np.float64))
        nimg = m.size // (3 * ny * nx)
        out = np.empty_like(m)
        be = np.ascontiguousarray(np.asarray(b_ext, dtype=np.float64).reshape(nimg, 3))
        mp = None
        if mask is not None:
            mk = np.ascontiguousarray(np.asarray(mask).reshape(-1).astype(np.uint8))
            mp = mk.ctypes.data_as(C.c_void_p)
        _check(lib().llg_warmstart_forward(self.h, nimg, int(ny), int(nx), _dp(m), mp, _dp(be), _dp(out)))
        return out


class WarmStartTrainer:
    """Training of the warm-start network on the GPU by this library's tensor-core
    kernels (forward, input gradient, weight gradient) with Adam on FP32 master
    weights.  Minibatches are device pointers (integers, e.g. torch tensors'
    data_ptr()): m0 and target FP32 SoA planes [nimg][3][ny][nx], mask uint8
    [nimg][ny][nx] or 0, bext float64 [nimg][3]."""

    def __init__(self, params, max_cells, device=0):
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float32).reshape(-1))
        h = C.c_void_p()
        _check(lib().llg_wstrain_create(_ctx(device), p.ctypes.data_as(C.POINTER(C.c_float)), p.size,
                                        int(max_cells), C.byref(h)))
        self.h = h
        self.n = p.size

    def close(self):
        if getattr(self, "h", None):
            lib().llg_wstrain_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_spin_limit(self, polls):
        _check(lib().llg_wstrain_set_spin_limit(self.h, int(polls)))

    def gradients(self, nimg, ny, nx, m0_ptr, mask_ptr, bext_ptr, target_ptr):
        """(mean loss, gradient of the mean loss in the parameter layout); parameters unchanged."""
        loss = C.c_double()
        g = np.empty(self.n, dtype=np.float32)
        _check(lib().llg_wstrain_gradients(self.h, int(nimg), int(ny), int(nx), m0_ptr, mask_ptr or None, bext_ptr,
                                           target_ptr, C.byref(loss), g.ctypes.data_as(C.POINTER(C.c_float))))
        return loss.value, g

    def step(self, nimg, ny, nx, m0_ptr, mask_ptr, bext_ptr, target_ptr, lr, beta1=0.9, beta2=0.999, eps=1e-8,
             read_loss=True):
        """One Adam step; returns the minibatch's mean loss (None with read_loss=False: no synchronisation)."""
        loss = C.c_double()
        _check(lib().llg_wstrain_step(self.h, int(nimg), int(ny), int(nx), m0_ptr, mask_ptr or None, bext_ptr,
                                      target_ptr, float(lr), float(beta1), float(beta2), float(eps),
                                      C.byref(loss) if read_loss else None))
        return loss.value if read_loss else None

    def sync(self):
        _check(lib().llg_wstrain_sync(self.h))

    def params(self):
        out = np.empty(self.n, dtype=np.float32)
        _check(lib().llg_wstrain_get_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out


def init_random(n, seed):
    """init_random (initial_states.rs:59-68)."""
    out = np.empty((int(n), 3))
    lib().llg_init_random(int(n), C.c_uint64(seed), _dp(out))
    return out


def init_uniform_with_noise(n, direction, noise, seed, m=None):
    """init_uniform_with_noise (initial_states.rs:43-56); zero cells of `m` are skipped."""
    out = np.ones((int(n), 3)) if m is None else np.ascontiguousarray(m, dtype=np.float64).copy()
    d = np.ascontiguousarray(np.asarray(direction, dtype=np.float64).reshape(3))
    lib().llg_init_uniform_with_noise(int(n), _dp(d), float(noise), C.c_uint64(seed), _dp(out))
    return out
