"""In-tree build of libbbrt_cuda.so for sm_100a.

    python -m billardballraytracing3d_b200.build [--force]

CUDA sources are compiled by nvcc for sm_100a only (-gencode
arch=compute_100a,code=sm_100a).  Kernels whose decisions must match the
reference bit for bit (trace_kernels.cu) are compiled with -fmad=false; host
C++ is compiled with -ffp-contract=off for the same reason.  Objects and the
library are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbbrt_cuda.so")
INCLUDE = os.path.normpath(os.path.join(HERE, "..", "include"))
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# per-source extra flags
CU_FLAGS = {
    "trace_kernels.cu": ["-fmad=false"],
    "scene_compile.cu": ["-fmad=false"],
}


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(CSRC, "*.hpp")) + glob.glob(os.path.join(INCLUDE, "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        name = os.path.basename(src)
        obj = os.path.join(BUILD, name + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs + [__file__]):
            _run([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                  "--expt-relaxed-constexpr", *CU_FLAGS.get(name, []), "-I", INCLUDE, "-c", src, "-o", obj], verbose)
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))):
        name = os.path.basename(src)
        obj = os.path.join(BUILD, name + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs + [__file__]):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-Wall",
                  "-I", os.path.join(CUDA_HOME, "include"), "-I", INCLUDE, "-c", src, "-o", obj], verbose)
    if force or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        _run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-Xcompiler", "-fopenmp", "-lgomp"], verbose)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
