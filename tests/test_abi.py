"""CPU checks of the C ABI library: it loads, exports every symbol the header
declares, reports errors through statuses, and its host-side input generators
match the oracle bit for bit.  No GPU compute is called here."""
import ctypes as C
import os

import numpy as np


def test_library_exports_every_declared_symbol(gpu):
    names = gpu.declared_symbols()
    assert len(names) >= 20
    lib = C.CDLL(gpu.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version(gpu):
    assert gpu.lib().llg_abi_version() == 2


def test_errors_are_statuses_not_aborts(gpu):
    import torch

    h = C.c_void_p()
    rc = gpu.lib().llg_ctx_create(-1 if torch.cuda.is_available() else 0, C.byref(h))
    assert rc in (-1, -6)  # LLG_ERR_INVALID / LLG_ERR_NO_DEVICE
    assert len(gpu.last_error()) > 0


def test_init_generators_match_oracle(gpu, orc):
    assert np.array_equal(gpu.init_random(500, 77), orc.init_random(500, 77))
    base = np.ones((64, 3))
    base[::7] = 0.0
    assert np.array_equal(gpu.init_uniform_with_noise(64, (0, 1, 1), 0.1, 5, base),
                          orc.init_uniform_with_noise(64, (0, 1, 1), 0.1, 5, base))


def test_default_relax_settings_match_oracle(gpu, orc):
    a = gpu.RelaxSettings.default()
    b = orc.default_relax_settings()
    for name, _ in gpu.RelaxSettings._fields_:
        assert getattr(a, name) == getattr(b, name), name


def test_default_minimize_settings_match_oracle(gpu, orc):
    a = gpu.MinimizeSettings.default()
    b = orc.default_minimize_settings()
    for name, _ in gpu.MinimizeSettings._fields_:
        assert getattr(a, name) == getattr(b, name), name
    # MinimizeSettings::default (minimize.rs:65-92)
    assert (a.torque_threshold, a.max_iters, a.lambda0, a.dm_stop, a.dm_samples) == (5e-4, 20000, 2e-2, 1e-6, 10)
    assert a.has_dm_stop and a.has_dm_torque_gate and a.has_dm_torque_gate_max
    assert C.sizeof(gpu.MinimizeSettings) == 136 and C.sizeof(gpu.MinimizeReport) == 56


def test_warmstart_param_count_matches_reference_layout(gpu):
    import warmstart_ref

    assert gpu.WarmStartNet.param_count() == warmstart_ref.param_count() == 39907


def test_demag_cache_filename_matches_reference_naming(gpu):
    g = gpu.Grid2D(128, 32, 4e-9, 4e-9, 3e-9)
    assert gpu.demag_cache_filename(g, 0, 0) == (
        "out/demag_cache/demag_kernel_nx128_ny32_pbcx0_pbcy0_px256_py64_dx4.000e-9_dy4.000e-9_dz3.000e-9_acc10.00.bin")
    g = gpu.Grid2D(2, 128, 1e-9, 1e-9, 0.5e-9)
    assert gpu.demag_cache_filename(g, 32, 0) == (
        "out/demag_cache/demag_kernel_nx2_ny128_pbcx32_pbcy0_px2_py256_dx1.000e-9_dy1.000e-9_dz5.000e-10_acc10.00.bin")


def test_struct_layouts_match_header(gpu, tmp_path):
    """Every public struct of include/llg_b200.h, as the C compiler lays it out, has the
    size and field offsets of its ctypes mirror (the Rust #[repr(C)] structs of the
    integration guide follow the same rules)."""
    import subprocess

    mirrors = {"llg_grid": gpu._Grid, "llg_material": gpu._Material, "llg_params": gpu._Params,
               "llg_relax_settings": gpu.RelaxSettings, "llg_relax_report": gpu.RelaxReport,
               "llg_minimize_settings": gpu.MinimizeSettings, "llg_minimize_report": gpu.MinimizeReport,
               "llg_energy_breakdown": gpu.EnergyBreakdown, "llg_amr_patch": gpu._AmrPatch,
               "llg_ovf_meta": gpu._OvfMeta}
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "llg_b200.h"', "int main(void) {"]
    for cname, cls in mirrors.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, key, val = line.split()
        got[(cname, key)] = int(val)
    for cname, cls in mirrors.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_trainer_parameter_layout_matches_the_network():
    import warmstart_train as T

    p = T.init_params(3)
    assert p.dtype == np.float32 and p.size == sum(co * 9 * ci + co for ci, co in T.LAYERS)
