"""The backprojectors' reciprocal (one Newton-Raphson step from rcp.approx,
jenhine_b200/csrc/bp_common.cuh) equals CUDA's correctly rounded __frcp_rn
for every float whose reciprocal is normal: tests/cuda/reciprocal_check.cu,
built here with nvcc for sm_100a and run over all 4.23e9 such values."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_newton_raphson_reciprocal_is_correctly_rounded(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = str(tmp_path / "reciprocal_check")
    src = os.path.join(ROOT, "tests", "cuda", "reciprocal_check.cu")
    inc = os.path.join(ROOT, "jenhine_b200", "csrc")
    b = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-I", inc,
                        src, "-o", exe], capture_output=True, text=True, timeout=300)
    assert b.returncode == 0, b.stdout + b.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "mismatches 0" in r.stdout, r.stdout + r.stderr
