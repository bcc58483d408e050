"""Builds the in-tree CUDA library and the drop-in CLI for sm_100a.

    python marineseis-fdm-2d_b200/builder.py

Outputs (git-ignored, shipped with the tree): libmfdm.so next to this file
and bin/main_debug. Rebuilds only when a source is newer than its output.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libmfdm.so")
CLI = os.path.join(HERE, "bin", "main_debug")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC"] + ARCH


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    """Compiles libmfdm.so and bin/main_debug; returns the library path."""
    nvcc = _nvcc()
    deps = _sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    deps.append(os.path.join(ROOT, "include", "mfdm.h"))
    lib_srcs = [s for s in _sources() if not s.endswith("main_debug.cpp")]
    if force or _stale(LIB, deps):
        cmd = [nvcc] + NVCC_FLAGS + ["-shared", "-o", LIB] + lib_srcs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    if force or _stale(CLI, [LIB, os.path.join(CSRC, "main_debug.cpp")]):
        cmd = [nvcc] + ARCH + ["-O2", "-std=c++17", os.path.join(CSRC, "main_debug.cpp"), "-L" + HERE,
               "-lmfdm", "-Xlinker", "-rpath=$ORIGIN/..", "-o", CLI]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
