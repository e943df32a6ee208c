"""Builds the in-tree CUDA library code_only_b200/_lib/libsfmg.so for sm_100a.

    python -m code_only_b200.build [--force]

nvcc compiles every source of csrc/ into one shared library with
-gencode arch=compute_100a,code=sm_100a.  --fmad=false keeps a*b+c as two
rounded operations so that FP64 results equal the reference's expression
order bit for bit; the kernels are bandwidth bound, so nothing is lost.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libsfmg.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "--fmad=false", "-lineinfo",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "-Xcompiler", "-fopenmp", "-lgomp",   # host threads of the host-array call's staging
    "-shared",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cuh", ".h"))]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = _sources() + [os.path.join(INCLUDE, "sfmg.h"), os.path.abspath(__file__)]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = True) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    units = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith(".cu")]
    tmp = LIB + ".tmp"
    cmd = [_nvcc()] + NVCC_FLAGS + ["-I", INCLUDE, "-o", tmp] + units
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
