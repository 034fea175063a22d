"""The allocation-free demag entry point, for callers that cannot allocate
device memory where they need the field (a framework whose pool owns every
device allocation, a real-time loop, code where cudaMalloc is not allowed).

It is checked through the C ABI against the CPU FP64 oracle (the oracle's own
kernel planes are passed in) and against llg_compute_demag_field, the regular
entry point, on two calls in a row (the static scratch is shared between calls).
Sizes cover small films, the largest square film the scratch holds (1024 x 1024),
a near-maximum non-square film (2048 x 600) and prime lengths (97 x 61), which take
the generic DFT pass.  This file is collected last on purpose."""
import numpy as np
import pytest

from helpers import case, gpu_solver, oracle_solver, random_m, rel_err

pytestmark = pytest.mark.gpu

TOL_FP32 = 2e-5  # same tolerance as the other FP32 field parity tests


def _call(gpu, nx, ny, ms, m, planes):
    import torch

    b_dev = torch.empty((3, ny, nx), dtype=torch.float32, device="cuda")
    m_dev = torch.from_numpy(np.ascontiguousarray(m.T.reshape(3, ny, nx))).to(torch.float32).to("cuda")
    stream = torch.cuda.current_stream()
    gpu.demag_field_noalloc(nx, ny, ms, m_dev.data_ptr(), planes.data_ptr(), b_dev.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    return b_dev.cpu().numpy().reshape(3, nx * ny).T


@pytest.mark.parametrize("nx,ny", [(64, 32), (97, 61), (256, 256), (1024, 1024)])
def test_noalloc_demag_matches_oracle(orc, gpu, nx, ny):
    import torch

    c = case(nx, ny)
    o = oracle_solver(orc, c)
    ko = o.kernel_kspace()   # [4, 2ny, 2nx] complex, unscaled
    planes = torch.from_numpy(np.ascontiguousarray(ko[:, : ny + 1, : nx + 1].real)).to("cuda")
    for call, seed in enumerate((11, 12)):
        m = random_m(orc, nx * ny, seed + nx)
        b = _call(gpu, nx, ny, c["ms"], m, planes)
        assert rel_err(b, o.demag_field(m)) <= TOL_FP32, call


@pytest.mark.parametrize("nx,ny", [(64, 32), (96, 40), (2048, 600)])
def test_noalloc_demag_matches_regular_entry_point(orc, gpu, nx, ny):
    import torch

    c = case(nx, ny)
    ref = gpu_solver(gpu, c, gpu.FP32)
    planes = torch.from_numpy(np.ascontiguousarray(ref.kernel_kspace())).to("cuda")
    for call, seed in enumerate((11, 12)):
        m = random_m(orc, nx * ny, seed + nx)
        ref.set_state(m)
        b = _call(gpu, nx, ny, c["ms"], m, planes)
        assert rel_err(b, ref.compute_demag_field()) <= TOL_FP32, call


def test_noalloc_rejects_oversized_film(gpu):
    import torch

    x = torch.zeros(16, dtype=torch.float32, device="cuda")
    with pytest.raises(gpu.LLGError) as e:
        gpu.demag_field_noalloc(2048, 2048, 8e5, x.data_ptr(), x.data_ptr(), x.data_ptr())
    assert "32 MiB" in str(e.value)
