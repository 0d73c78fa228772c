"""Builds libsolunar_fluid.so in-tree for sm_100a.

Kernels are compiled with -fmad=false and IEEE division and square root (nvcc's defaults
without --use_fast_math), so every expression rounds as the reference's scalar f32 code.  The
CUDA runtime is linked statically so the library does not depend on which libcudart another
module of the process (torch) loaded first.

    python -m solunar_b200.build [--verbose]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsolunar_fluid.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# kernels whose rounding follows the reference: no contraction, IEEE division and square root
CUDA_SOURCES = ["kernels.cu", "noalloc.cu"]
# the FAST arithmetic variants: contraction on
CUDA_FAST_SOURCES = ["kernels_fast.cu", "adjoint.cu"]
HOST_SOURCES = ["world_core.cpp", "world_walls.cpp", "world_bodies.cpp", "world_substep.cpp", "world_adjoint.cpp",
                "world_flows.cpp", "world_snapshot.cpp", "capi.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    # the system compiler; the image may point CXX at a wrapper
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _cuda_include() -> str:
    return os.path.join(os.path.dirname(os.path.dirname(_nvcc())), "include")


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "solunar_fluid.h"))
    objects = []
    nvcc = _nvcc()
    for src in CUDA_SOURCES + CUDA_FAST_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objects.append(obj)
        if force or _stale(obj, [path] + headers):
            rounding = (["-fmad=true"] if src in CUDA_FAST_SOURCES else
                        ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"])
            cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", *rounding, "--extended-lambda", "-Xcompiler",
                   "-fPIC", "-I", CSRC, "-c", path, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            subprocess.run(cmd, check=True)
    for src in HOST_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objects.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [_cxx(), "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
                   "-Wno-unused-function", "-I", _cuda_include(), "-I", CSRC, "-c", path, "-o", obj]
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objects):
        cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objects]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(LIB)
