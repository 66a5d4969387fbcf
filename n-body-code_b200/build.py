"""Builds libnbody_cuda.so (sm_100a) in-tree, plus the C++ driver.

    python n-body-code_b200/build.py [--force] [--verbose]

Outputs (git-ignored, shipped with the source tree):
    n-body-code_b200/lib/libnbody_cuda.so   the C-ABI of include/nbody_cuda.h
    n-body-code_b200/lib/nbody_app           the --N/--Ncycle driver
nvcc links the CUDA runtime statically, so the library does not depend on
the runtime version that other libraries in the process (torch) bring.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libnbody_cuda.so")
APP = os.path.join(LIB_DIR, "nbody_app")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-ccbin", "/usr/bin/g++"]

LIB_SOURCES = ["engine.cu", "peaks.cu", "noalloc.cu", "ensemble.cu", "adjoint.cu", "ic.cpp", "state_io.cpp"]


def _sources(names, base):
    return [os.path.join(base, s) for s in names if os.path.exists(os.path.join(base, s))]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    out = [os.path.join(ROOT, "include", "nbody_cuda.h")]
    for d in (CSRC, HOST):
        if os.path.isdir(d):
            out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".cuh", ".h"))]
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = _sources(LIB_SOURCES, CSRC)
    if force or _newer(LIB, srcs + _headers()):
        cmd = [NVCC, *ARCH, *CUFLAGS, "-shared", "-o", LIB, *srcs]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    host_srcs = _sources(["main.cpp", "nbody_gpu.cpp"], HOST)
    if len(host_srcs) == 2 and (force or _newer(APP, host_srcs + _headers() + [LIB])):
        cmd = ["/usr/bin/g++", "-std=c++17", "-O2", f"-I{os.path.join(ROOT, 'include')}",
               "-o", APP, *host_srcs, f"-L{LIB_DIR}", "-lnbody_cuda", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    sys.exit(0)
