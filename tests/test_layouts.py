"""Index algebra of the register-FFT kernels, checked on the host from the kernels' own
headers (tests/harness/layout_checks.cu, built with nvcc as host code; no GPU): the
register caps per resident-block count, the parity-split kernel columns read by the
column pass, and the swizzled slots of the staged spectrum (permutation, per-thread
affine addressing, shared-memory wavefronts of a warp's reads)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_layout_index_algebra(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = tmp_path / "layout_checks"
    subprocess.run([nvcc, "-std=c++17", "-O1", "-x", "cu", "-gencode", "arch=compute_100a,code=sm_100a", "-I", os.path.join(ROOT, "llg-sim_b200", "csrc"),
                    os.path.join(HERE, "harness", "layout_checks.cu"), "-o", str(exe)],
                   check=True, capture_output=True, timeout=600)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip().endswith("ok"), out.stdout + out.stderr
