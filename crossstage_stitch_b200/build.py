"""Builds libstitch_b200.so in place for sm_100a.

    python -m crossstage_stitch_b200.build [--force]

Each .cu / .cpp under csrc/ is compiled by nvcc to an object (in parallel),
then linked into crossstage_stitch_b200/libstitch_b200.so with the CUDA
runtime linked statically, so the library needs only the driver at run time.
Objects are rebuilt when a source or any csrc header is newer.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libstitch_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: the S5 solver and every float stage formula are written as
# separately rounded operations; contraction into FMA would change results.
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "--extended-lambda",
              "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=default",
              "-I", str(CSRC), "-I", str(INCLUDE)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted([*CSRC.glob("*.cu"), *CSRC.glob("*.cpp")])


def newest_header() -> float:
    hs = [*CSRC.glob("*.cuh"), *CSRC.glob("*.hpp"), *CSRC.glob("*.inc"), *INCLUDE.glob("*.h")]
    return max((h.stat().st_mtime for h in hs), default=0.0)


def compile_one(src: Path, force: bool, header_time: float) -> Path:
    obj = BUILD / (src.stem + ".o")
    if (not force and obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime
            and obj.stat().st_mtime >= header_time):
        return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    header_time = newest_header()
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force, header_time), srcs))
    newest_obj = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest_obj:
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-Xlinker", "-Bsymbolic",
               *[str(o) for o in objs], "-o", str(LIB)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force))


if __name__ == "__main__":
    sys.exit(main())
