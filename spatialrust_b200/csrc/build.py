"""Builds spatialrust_b200/libsrcuda.so (the C ABI of include/srcuda.h) with nvcc for sm_100a.

Usage: python -m spatialrust_b200.csrc.build [--force] [--verbose-ptxas]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "libsrcuda.so")
SOURCES = [os.path.join(HERE, "srcuda.cu"), os.path.join(HERE, "server.cu")]
HEADERS = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith((".cuh", ".cu", ".h"))] + [
    os.path.join(ROOT, "include", "srcuda.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    # No fast math: the key, predicate and centroid arithmetic must round like
    # the reference's f32/f64 code.
    "-prec-div=true", "-prec-sqrt=true", "-fmad=true",
    "-Xcompiler", "-fPIC", "-shared",
    "-I", os.path.join(ROOT, "include"),
    "-lpthread",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in SOURCES + HEADERS)


def build(force: bool = False, ptxas_verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *NVCC_FLAGS, *(["-Xptxas", "-v"] if ptxas_verbose else []), "-o", tmp, *SOURCES]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, ptxas_verbose="--verbose-ptxas" in sys.argv)
    print(LIB)
