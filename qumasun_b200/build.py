"""Builds the engine's shared library (sm_100a) in-tree.

``python -m qumasun_b200.build`` compiles every ``csrc/*.cu`` with nvcc into
``qumasun_b200/libqumasun_b200.so`` (the C ABI of include/qumasun_b200.h).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libqumasun_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = (sources() + glob.glob(os.path.join(HERE, "csrc", "*.h")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh"))
            + glob.glob(os.path.join(ROOT, "include", "*.h")))
    return any(os.path.getmtime(f) > t for f in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"),
           *extra, "-o", LIB + ".tmp", *sources(),
           "-L/usr/local/cuda/lib64", "-lcublas", "-lcusolver", "-lcufft",
           "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
