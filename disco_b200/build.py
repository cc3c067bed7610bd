"""Build recipe of the native libraries (in-tree, so they travel with the repo).

  disco_b200/_lib/libdisco_b200.so   CUDA kernels for sm_100a + the C-ABI
                                     (include/disco_b200.h)
  disco_b200/_lib/libdisco_geom.so   host input synthesis (include/disco_geometry.h)
  disco_b200/_lib/libdisco_backend.so  C++ shim exposing the reference backend
                                     interface (kroupaGPU, gpuAvailable, ...)

nvcc cross-compiles for sm_100a without a GPU.  Each output is rebuilt only
when one of its sources is newer.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "_lib")
INC = os.path.join(REPO, "include")

NVCC = os.environ.get("DISCO_NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("DISCO_CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CUDA_SOURCES = ["field.cu", "field_fp32.cu", "batch.cu", "mlp.cu", "far.cu", "prismatic.cu", "lattice.cu", "writer.cu", "capi.cu"]
CUDA_HEADERS = ["common.cuh", "field.cuh", "field_device.cuh", "field_fp32.cuh", "tcgen05.cuh", "mlp.cuh"]

LIB_CUDA = os.path.join(LIB, "libdisco_b200.so")
LIB_GEOM = os.path.join(LIB, "libdisco_geom.so")
LIB_SHIM = os.path.join(LIB, "libdisco_backend.so")


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force=False, verbose=True, ptxas_info=False):
    os.makedirs(LIB, exist_ok=True)
    srcs = [os.path.join(CSRC, f) for f in CUDA_SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in CUDA_HEADERS] + \
        [os.path.join(INC, "disco_b200.h"), __file__]
    if force or _stale(LIB_CUDA, deps):
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-shared",
               "-Xcompiler", "-fPIC,-O3,-ffp-contract=off", "-I", INC, *srcs, "-o", LIB_CUDA]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        _run(cmd, verbose)
    geom = os.path.join(CSRC, "geometry.cpp")
    gdeps = [geom, os.path.join(INC, "disco_geometry.h"), os.path.join(INC, "disco_b200.h"), __file__]
    if force or _stale(LIB_GEOM, gdeps):
        # the reference's host flags (Code/Makefile:66) with a portable -march
        _run([CXX, "-std=c++17", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared",
              "-I", INC, geom, "-o", LIB_GEOM], verbose)
    shim = os.path.join(CSRC, "backend_shim.cpp")
    sdeps = [shim, os.path.join(INC, "backend.hpp"), os.path.join(INC, "disco_b200.h"), LIB_CUDA, __file__]
    if os.path.exists(shim) and (force or _stale(LIB_SHIM, sdeps)):
        _run([CXX, "-std=c++14", "-O2", "-fPIC", "-shared", "-I", INC, shim,
              "-L", LIB, "-ldisco_b200", "-Wl,-rpath,$ORIGIN", "-o", LIB_SHIM], verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
