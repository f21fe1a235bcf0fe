"""Builds libvsmc_cuda.so in-tree for sm_100a with nvcc.

    python -m vsmc_b200.build [--force]

The library is written for B200 only: every kernel is compiled for
``-gencode arch=compute_100a,code=sm_100a`` with ``-lineinfo``; there is no
other architecture and no fallback path.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib", "libvsmc_cuda.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
         "--expt-relaxed-constexpr"]
OBJ = os.path.join(HERE, "lib", "obj")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _inputs():
    return (sources() + glob.glob(os.path.join(CSRC, "*.cuh"))
            + glob.glob(os.path.join(ROOT, "include", "vsmc_b200", "*.cuh"))
            + [os.path.join(ROOT, "include", "vsmc_cuda.h")])


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every translation unit to an object (in parallel, one nvcc
    per source) and link the shared library."""
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, "-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd))
        objs.append(obj)
        procs.append((subprocess.Popen(cmd), cmd))
    failed = [cmd for p, cmd in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    tmp = LIB + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
