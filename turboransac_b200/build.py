"""Build step: compile libtbr.so for sm_100a, in-tree.

    python -m turboransac_b200.build

nvcc cross-compiles without a GPU, so this runs on any machine with CUDA 12.8+.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc", "tbr_engine.cu")
OUT = os.path.join(HERE, "libtbr.so")
DEPS = [os.path.join(HERE, "csrc", f) for f in ("tbr_engine.cu", "tbr_kernels.cuh", "tbr_device.cuh")] + [
    os.path.join(ROOT, "include", "tbr.h")]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "-cudart", "static", "-diag-suppress", "177,550"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in DEPS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    cmd = [nvcc(), *NVCC_FLAGS, "-o", OUT, SRC]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
