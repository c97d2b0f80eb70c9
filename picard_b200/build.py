"""Builds libpicard_gpu.so in-tree for sm_100a with nvcc.

particles_exact.cu is compiled with --fmad=false (the FP64 kernels keep the
reference's separately rounded multiplies and adds), and sort.cu too (its F64
sort key is the deposit's base-node expression); every other unit uses the
default contraction.  Objects go to picard_b200/_build/, the library to
picard_b200/lib/libpicard_gpu.so.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libpicard_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", SRC,
          "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]
UNITS = {
    "particles_exact.cu": ["--fmad=false"],
    "particles_fast.cu": [],
    "grid.cu": [],
    "bcpot_tc.cu": [],
    "solver.cu": [],
    "jacobi_resident.cu": [],
    "context.cu": [],
    "driver.cu": [],
    "server.cu": [],
    "batch.cu": [],
    "output.cu": [],
    "f90.cu": [],
    "sort.cu": ["--fmad=false"],
    "spectral.cu": [],
    "bcpot_fft.cu": [],
}


def _newer(dst: str, srcs: list[str]) -> bool:
    if not os.path.exists(dst):
        return False
    t = os.path.getmtime(dst)
    return all(os.path.getmtime(s) <= t for s in srcs)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    headers = [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith(".cuh")]
    headers += [os.path.join(ROOT, "include", h) for h in ("picard_gpu.h", "picard_server.h", "picard_io.h", "picard_f90.h")]
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(SRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if not force and _newer(obj, [src] + headers):
            continue
        cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or not _newer(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
