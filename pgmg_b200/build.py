"""Builds libpgmg_b200.so in-tree with nvcc for sm_100a.

    python -m pgmg_b200.build        (or build() from __graft_entry__)

The library is the product: CUDA kernels for sm_100a plus the C ABI declared
in include/pgmg_dev.h.  It is built in place (pgmg_b200/libpgmg_b200.so) so
that it travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libpgmg_b200.so")
OBJDIR = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp", "-I" + os.path.join(ROOT, "include")]

SOURCES = ["capi.cu", "batch.cu", "noalloc.cu", "problems.cpp"]


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    for s in src_list:
        if os.path.getmtime(s) > t:
            return True
    return False


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "pgmg_dev.h"))
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJDIR, os.path.splitext(s)[0] + ".o")
        objs.append(obj)
        if force or _newer([src] + headers, obj):
            cmd = [NVCC] + CUFLAGS + ["-c", src, "-o", obj]
            if s.endswith(".cpp"):
                cmd = [os.environ.get("CXX", "g++"), "-O3", "-std=c++17", "-fPIC", "-fopenmp",
                       "-I" + os.path.join(ROOT, "include"), "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _newer(objs, OUT):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lgomp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
