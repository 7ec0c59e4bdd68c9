"""Build recipe of libnca_b200.so (sm_100a) into nca_b200/ next to its Python front end.

    python nestedcrossapproximation.jl_b200/build.py [--force]

nvcc cross-compiles for sm_100a without a GPU. The host planner is compiled with
-ffp-contract=off (its arithmetic is reproduced bit for bit elsewhere); build_kernels.cu with
--fmad=false (the pivot search and the tree mimicry spell out every fused multiply-add).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUTDIR = os.path.join(HERE, "nca_b200")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(OUTDIR, "libnca_b200.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-ccbin", CXX, "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-mfma", "-I", INCLUDE, "-I", CSRC, "-pthread"]

UNITS = [
    ("host_plan.cpp", "cxx", []),
    ("directional.cpp", "cxx", []),
    ("build_kernels.cu", "nvcc", ["--fmad=false"]),
    ("mimicry.cu", "nvcc", ["--fmad=false"]),
    ("apply_kernels.cu", "nvcc", []),
    ("tc_gather.cu", "nvcc", []),
    ("tree_kernels.cu", "nvcc", ["--fmad=false"]),
    ("capi.cu", "nvcc", []),
]
HEADERS = ["nca_internal.h", "entry.cuh", "build_kernels.cuh", "apply_kernels.cuh"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "nca_b200.h")]
    objs = []
    for src, kind, extra in UNITS:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            if kind == "cxx":
                cmd = [CXX] + CXXFLAGS + ["-c", path, "-o", obj]
            else:
                cmd = [NVCC] + ARCH + NVFLAGS + extra + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", CXX, "-o", LIB] + objs + ["-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
