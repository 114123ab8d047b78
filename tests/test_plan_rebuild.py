"""Building a batch plan twice on one object gives a fresh plan's layout.
The check is a small host program (tests/plan_rebuild_check.cu) compiled
against the package's headers and linked to the built library; it creates
plans without a device (no pinned staging), so it runs on the CPU."""
import os
import shutil
import subprocess
import tempfile
from pathlib import Path

import pytest

from crossstage_stitch_b200 import build as native

ROOT = Path(__file__).resolve().parents[1]


def test_plan_build_twice_equals_fresh_plan():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not available")
    lib = native.build()
    with tempfile.TemporaryDirectory() as d:
        exe = Path(d) / "plan_rebuild_check"
        cmd = [nvcc, *native.ARCH, "-std=c++17", "-O1", "-I", str(native.CSRC), "-I", str(native.INCLUDE),
               str(ROOT / "tests" / "plan_rebuild_check.cu"), str(lib), "-o", str(exe),
               "-Xlinker", f"-rpath={lib.parent}"]
        built = subprocess.run(cmd, capture_output=True, text=True)
        assert built.returncode == 0, built.stderr[-4000:]
        env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
        out = subprocess.run([str(exe)], capture_output=True, text=True, env=env)
        assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
        assert "plan rebuild ok" in out.stdout
