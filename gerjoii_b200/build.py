"""Builds the sm_100a shared library in-tree (gerjoii_b200/_lib/libgerjoii_b200.so).

    python -m gerjoii_b200.build          # or gerjoii_b200.build.build()

nvcc cross-compiles for sm_100a without a GPU.  The library links only the
CUDA runtime (static) and cuFFT; it has no torch dependency.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libgerjoii_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    deps.append(os.path.join(os.path.dirname(HERE), "include", "gerjoii_gpu.h"))
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, out: str | None = None, defines=()) -> str:
    """Compiles the library; `out` and `defines` build a tuning variant elsewhere."""
    target = out or LIB
    if out is None and not force and up_to_date():
        return LIB
    os.makedirs(os.path.dirname(target), exist_ok=True)
    tmp = target + ".tmp"
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-cudart", "static", *[f"-D{d}" for d in defines], "-o", tmp, *sources(), "-lcufft"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(tmp, target)
    return target


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
