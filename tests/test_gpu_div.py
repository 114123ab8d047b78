"""The MSAC residual's shared-reciprocal division (Markstein's theorem) must
equal the plain division bit for bit: builds tests/gpu_div_check.cu with the
library's flags and checks 2^27 seeded random quotients and residuals."""
import shutil
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "crossstage_stitch_b200" / "csrc"
INCLUDE = HERE.parent / "include"


def test_shared_reciprocal_division_is_exact(cuda, tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "div_check"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-fmad=false", "-std=c++17",
                    "-I", str(CSRC), "-I", str(INCLUDE), str(HERE / "gpu_div_check.cu"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True, timeout=120).stdout
    assert out.split() == ["inputs", str(1 << 27), "mismatch", "0"], out
