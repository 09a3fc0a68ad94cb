"""Builds the engine's shared library in-tree for sm_100a.

The library (``mercurydpm_fork_b200/libdem_b200.so``) exports the C ABI of
``include/dem_b200.h``. It is compiled with ``--fmad=false`` so that every
FP64 expression is evaluated as separately rounded IEEE operations, the same
way the reference's x86-64 build evaluates it.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdem_b200.so")
# the calibration surrogate (tensor-core MLP) is a library of its own; it is
# built without --fmad=false (no reference arithmetic to reproduce)
SURROGATE_LIB = os.path.join(HERE, "libdem_surrogate.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-O2", "-shared",
         "-cudart", "static"]


def sources():
    return [os.path.join(CSRC, "dem_engine.cu")]


def surrogate_sources():
    return [os.path.join(CSRC, "surrogate.cu")]


def headers():
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cuh", ".h")):
                out.append(os.path.join(d, f))
    return out


def needs_build(lib: str = LIB, srcs=None) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(os.path.getmtime(f) > t for f in (srcs or sources()) + headers() + [__file__])


def _compile(lib: str, srcs, flags, verbose: bool):
    cmd = [NVCC, *ARCH, *flags, "-I", os.path.join(ROOT, "include"), *srcs, "-o", lib + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(lib + ".tmp", lib)


def build(force: bool = False, verbose: bool = False) -> str:
    if force or needs_build(LIB, sources()):
        _compile(LIB, sources(), FLAGS, verbose)
    if force or needs_build(SURROGATE_LIB, surrogate_sources()):
        _compile(SURROGATE_LIB, surrogate_sources(), [f for f in FLAGS if f != "--fmad=false"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
