"""In-tree build of the native libraries (run by __graft_entry__.build()).

* libfvmhd3d_b200.so : the sm_100a CUDA kernels and the C-ABI
  (nvcc -gencode arch=compute_100a,code=sm_100a)
* libfvmmesh.so      : the host Voronoi mesh builder (g++ -fopenmp)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build_cuda(force=False):
    out = os.path.join(HERE, "libfvmhd3d_b200.so")
    srcs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h"))]
    srcs.append(os.path.join(HERE, "..", "include", "fvmhd3d_b200.h"))
    if force or _stale(out, srcs):
        _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
              "-diag-suppress", "177", "-o", out, os.path.join(CSRC, "fvm_kernels.cu"),
              os.path.join(CSRC, "fvm_fused.cu")])
    return out


def build_mesh(force=False):
    out = os.path.join(HERE, "libfvmmesh.so")
    src = os.path.join(CSRC, "voronoi.cpp")
    if force or _stale(out, [src]):
        _run(["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-o", out, src])
    return out


def build_all(force=False):
    build_mesh(force)
    build_cuda(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
