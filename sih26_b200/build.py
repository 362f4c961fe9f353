"""Builds the CUDA library in-tree: sih26_b200/_lib/libsankhya_pdhg_gpu.so (sm_100a only).

`python -m sih26_b200.build` or `build_library()`; nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIBNAME = "libsankhya_pdhg_gpu.so"
LIBPATH = os.path.join(LIBDIR, LIBNAME)

SOURCES = ["pdhg_solver.cu", "pdhg_host.cpp", "residuals_noalloc.cu", "batch_server.cu",
           "wire.cpp", "qp_solver.cu"]
HEADERS = ["device_common.cuh", "pdhg_kernels.cuh", "pdhg_host.cuh", "batch_kernels.cuh",
           "prep_kernels.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newest_input() -> float:
    paths = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    paths.append(os.path.join(ROOT, "include", "sankhya_pdhg_gpu.h"))
    return max(os.path.getmtime(p) for p in paths)


def build_library(force: bool = False, verbose: bool = False) -> str:
    """Compiles the library when a source is newer than it; returns its path."""
    if not force and os.path.exists(LIBPATH) and os.path.getmtime(LIBPATH) >= _newest_input():
        return LIBPATH
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = LIBPATH + ".tmp"
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp",
           "-shared", "-lgomp",
           "-Xptxas", "-v" if verbose else "-O3",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           *[os.path.join(CSRC, s) for s in SOURCES], "-o", tmp]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + proc.stdout + proc.stderr)
    if verbose:
        sys.stdout.write(proc.stdout + proc.stderr)
    os.replace(tmp, LIBPATH)
    return LIBPATH


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose="-v" in sys.argv))
