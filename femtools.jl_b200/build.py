"""Build libfemtools_b200.so in-tree with nvcc for sm_100a.

Usage: python femtools.jl_b200/build.py [--verbose-ptxas]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libfemtools_b200.so")
BUILD = os.path.join(HERE, "_build")
SOURCES = ["api.cu", "stokes3d.cu", "stokes3d_pipe.cu", "stokes3d_incr.cu", "adjoint3d.cu", "conv_bf16.cu", "warmstart_fields.cu", "geometry.cu", "postprocess.cu", "cellpressure.cu", "jacobian3d.cu", "simple.cu", "node.cu", "cap.cu", "coloring.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-rdc=true"]


def _stale(obj, src_files):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(s) > t for s in src_files)


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(HERE, "..", "include", "femtools_b200.h"))
    objs = []
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if force or verbose_ptxas or _stale(o, [s] + headers):
            cmd = [NVCC, *FLAGS, *extra, "-c", s, "-o", o]
            subprocess.check_call(cmd)
    if force or _stale(OUT, objs):
        subprocess.check_call([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
                               *objs, "-o", OUT, "-lcudart"])
    return OUT


if __name__ == "__main__":
    print(build(verbose_ptxas="--verbose-ptxas" in sys.argv, force="--force" in sys.argv))
