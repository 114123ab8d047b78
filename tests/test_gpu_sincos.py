"""The S3 orientation step takes cos and sin of its angle from one sincos()
call; that is only the reference's cos()/sin() result if the two agree bit
for bit on every angle it can produce. This builds a small CUDA program with
the library's flags and checks all 1,086,918,650 floats in [0, 6.2832]."""
import shutil
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent


def test_sincos_equals_sin_and_cos_on_every_angle(cuda, tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "sincos_check"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-fmad=false",
                    str(HERE / "gpu_sincos_check.cu"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True, timeout=120).stdout
    assert out.split() == ["inputs", "1086918650", "mismatch", "0"], out
