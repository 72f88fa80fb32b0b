"""Build recipe of libcathode_b200.so (sm_100a).

Compiles every CUDA source under csrc/ with nvcc for sm_100a into one shared
library next to this file.  The library is the product's C ABI
(include/cathode_b200.h); Python reaches it through ctypes (capi.py).
"""
from __future__ import annotations

import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libcathode_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
         "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def headers():
    return (sorted(glob.glob(os.path.join(HERE, "csrc", "*.h"))) +
            sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) +
            sorted(glob.glob(os.path.join(HERE, "..", "include", "*.h"))))


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in sources() + headers())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    cmd = [NVCC] + ARCH + FLAGS + ["-I", os.path.join(HERE, "..", "include")] + sources() + ["-o", LIB]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    import sys
    build(force=True, verbose="-v" in sys.argv)
    print(LIB)
