"""CPU checks of the C ABI library: it loads, exports every symbol the header
declares, reports errors through statuses, and its host-side input generators
match the oracle bit for bit.  No GPU compute is called here."""
import ctypes as C

import numpy as np


def test_library_exports_every_declared_symbol(gpu):
    names = gpu.declared_symbols()
    assert len(names) >= 20
    lib = C.CDLL(gpu.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version(gpu):
    assert gpu.lib().llg_abi_version() == 1


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
