"""Builds the native library of the package: libve.so (host C++ scene layer +
sm_100a CUDA kernels + the C ABI of include/ve.h), in-tree next to this file.

    python voxelengine3.0_b200/build.py [--force]

The CUDA translation unit is compiled with --fmad=false and IEEE division /
square root: the traversal and shading arithmetic must agree bit for bit with
the scalar CPU restatement used as the test oracle.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libve.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
                     "-ftz=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
                     "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-pthread"]

CU_SOURCES = ["render.cu"]
CXX_SOURCES = ["host/octree_cpu.cpp", "host/terrain.cpp", "host/host_api.cpp"]
HEADERS = ["ve_device.cuh", "raycast.cuh", "serve.cuh", "tc.cuh", "nrc.cuh", "nrc_host.cuh", "builder.cuh",
           "emissive.cuh", "lbuffer.cuh",
           "host/scene_host.h"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "ve.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _newer(o, [s] + headers):
            cmd = [NVCC] + CUDA_FLAGS + inc + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
        objs.append(o)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _newer(o, [s] + headers):
            cmd = ["g++"] + CXX_FLAGS + inc + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
        objs.append(o)
    if force or _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
