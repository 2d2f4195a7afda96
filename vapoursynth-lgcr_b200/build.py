"""Build the B200 Recon library in-tree.

    python vapoursynth-lgcr_b200/build.py [--force]

Compiles csrc/*.cu for sm_100a (nvcc -gencode arch=compute_100a,code=sm_100a,
-fmad=false so device arithmetic rounds like the reference's x86-64 scalar
build) and csrc/geometry.cpp with the host compiler (no FP contraction), and
links lgcr/liblgcr_b200.so. Objects go to _build/ (git-ignored).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "lgcr", "liblgcr_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-fmad=false", "-lineinfo", "-Xcompiler", "-fPIC",
                  "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off"]


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "lgcr_b200.h"))
    objects = []
    for name in sorted(os.listdir(CSRC)):
        src = os.path.join(CSRC, name)
        if name.endswith(".cu"):
            obj = os.path.join(BUILD, name[:-3] + ".o")
            if force or _newer([src] + headers, obj):
                extra = ["-Xptxas", "-v"] if verbose_ptxas else []
                _run([NVCC] + NVFLAGS + extra + ["-c", src, "-o", obj])
            objects.append(obj)
        elif name.endswith(".cpp"):
            obj = os.path.join(BUILD, name[:-4] + ".o")
            if force or _newer([src] + headers, obj):
                _run([CXX] + CXXFLAGS + ["-c", src, "-o", obj])
            objects.append(obj)
    if force or _newer(objects, OUT):
        _run([NVCC] + ARCH + ["-shared", "-o", OUT] + objects + ["-lpthread"])
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv)
