"""Build recipe of the oracle (test infrastructure only).

Three shared libraries, all host code:

  oracle/_build/libdisco_oracle.so        the CPU restatement, compiled with the
                                           reference's flags (-O3 -fopenmp, FMA
                                           contraction left on, Code/Makefile:66)
  oracle/_build/libdisco_oracle_nofma.so  the same with -ffp-contract=off: the
                                           pinned build the atom-set checks use
  oracle/_ref/libdisco_ref.so             the reference's own backend_cpu.cpp,
                                           loop.cpp and prismatic.cpp compiled in
                                           place from the reference tree, plus
                                           oracle/ref_harness.cpp; built only where
                                           the reference tree exists
  oracle/_ref/libdisco_ref_nofma.so       the same with -ffp-contract=off
  oracle/_ref/libdisco_ref_cuda.so        the reference's own CUDA backend
                                           (Code/backend_cuda.cu) compiled in place
                                           with nvcc for sm_100a and the
                                           Makefile's flags (Code/Makefile:67),
                                           plus oracle/ref_gpu_harness.cpp: the
                                           reference's GPU kernels, timed beside
                                           this library's on the same B200
  oracle/_ref/exec_b200                   the reference's own driver (Code/main.cpp
                                           and its host sources, Code/Makefile's
                                           SRC_HOST) compiled in place with
                                           -DWITH_CUDA and linked with this
                                           library's backend shim instead of
                                           backend_cuda.cu; yaml-cpp, absent here,
                                           is replaced by oracle/yaml_subset

GCC contracts a*b+c into FMAs where it sees fit, and it does not contract the
reference and the restatement identically (the reference folds nu = 0.35 at
compile time).  The contract-off builds of both are bit-identical; the
difference between the two default builds is the rounding floor of the
comparison, reported by the tests.

`-march=x86-64-v3` replaces the reference's `-march=native` so that the
libraries built here also run on the GPU host (AVX2 + FMA); both the reference
and the restatement get the same flags, which is what bit-identity needs.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
# The reference's Code/ directory: DISCO_REFERENCE_CODE, or the `reference`
# argument of build().  Unset: the reference's own libraries are not rebuilt
# (a prebuilt oracle/_ref is used where one exists).
REF_CODE = os.environ.get("DISCO_REFERENCE_CODE", "")

CXX = os.environ.get("DISCO_CXX", "g++")
BASE = ["-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared"]

ORACLE_SO = os.path.join(HERE, "_build", "libdisco_oracle.so")
ORACLE_NOFMA_SO = os.path.join(HERE, "_build", "libdisco_oracle_nofma.so")
REF_SO = os.path.join(HERE, "_ref", "libdisco_ref.so")
REF_NOFMA_SO = os.path.join(HERE, "_ref", "libdisco_ref_nofma.so")
REF_EXEC = os.path.join(HERE, "_ref", "exec_b200")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libdisco_ref_cuda.so")
NVCC = os.environ.get("DISCO_NVCC", "/usr/local/cuda/bin/nvcc")
HOST_SOURCES = ("main.cpp", "input.cpp", "loop.cpp", "loop_deform.cpp", "prismatic.cpp", "polycrystal.cpp",
                "twin.cpp", "backend_cpu.cpp")


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force=False, verbose=True, reference=None):
    global REF_CODE
    if reference:
        REF_CODE = reference
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    src = os.path.join(HERE, "disco_oracle.cpp")
    hdr = os.path.join(REPO, "include", "disco_b200.h")
    if force or _stale(ORACLE_SO, [src, hdr, __file__]):
        _run([CXX, "-std=c++17", *BASE, src, "-o", ORACLE_SO])
    if force or _stale(ORACLE_NOFMA_SO, [src, hdr, __file__]):
        _run([CXX, "-std=c++17", *BASE, "-ffp-contract=off", src, "-o", ORACLE_NOFMA_SO])
    if REF_CODE and os.path.isdir(REF_CODE):
        os.makedirs(os.path.join(HERE, "_ref"), exist_ok=True)
        harness = os.path.join(HERE, "ref_harness.cpp")
        ref_srcs = [os.path.join(REF_CODE, f) for f in ("backend_cpu.cpp", "loop.cpp", "prismatic.cpp")]
        ref_hdrs = [os.path.join(REF_CODE, f) for f in
                    ("backend.hpp", "barnett.hpp", "kroupa.hpp", "lattice.hpp", "loop.hpp", "prismatic.hpp")]
        deps = [harness, hdr, __file__, *ref_srcs, *ref_hdrs]
        if force or _stale(REF_SO, deps):
            _run([CXX, "-std=c++14", *BASE, "-I", REF_CODE, harness, *ref_srcs, "-o", REF_SO])
        if force or _stale(REF_NOFMA_SO, deps):
            _run([CXX, "-std=c++14", *BASE, "-ffp-contract=off", "-I", REF_CODE, harness, *ref_srcs,
                  "-o", REF_NOFMA_SO])
        build_driver(force)
        build_cuda(force)
    elif verbose:
        print("reference sources not given (DISCO_REFERENCE_CODE): oracle/_ref not rebuilt", flush=True)


def build_driver(force=False):
    """The reference's driver, unchanged, on this library's backend (the
    integration a maintainer would make, built here as a test harness)."""
    lib = os.path.join(REPO, "disco_b200", "_lib")
    shim = os.path.join(lib, "libdisco_backend.so")
    if not os.path.exists(shim):
        return
    srcs = [os.path.join(REF_CODE, f) for f in HOST_SOURCES]
    yaml_h = os.path.join(HERE, "yaml_subset", "yaml-cpp", "yaml.h")
    hdrs = [os.path.join(REF_CODE, f) for f in os.listdir(REF_CODE) if f.endswith(".hpp")]
    if force or _stale(REF_EXEC, [*srcs, *hdrs, yaml_h, shim, __file__]):
        _run([CXX, "-std=c++14", "-O3", "-march=x86-64-v3", "-fopenmp", "-DWITH_CUDA",
              "-I", os.path.join(HERE, "yaml_subset"), "-I", REF_CODE, *srcs,
              "-L", lib, "-ldisco_backend", "-ldisco_b200", "-Wl,-rpath,$ORIGIN/../../disco_b200/_lib",
              "-o", REF_EXEC])


def build_cuda(force=False):
    """The reference's CUDA backend for sm_100a: Code/backend_cuda.cu with
    the flags of Code/Makefile:67 (nvcc -O3 -std=c++14 -DWITH_CUDA, its
    default FMA contraction), -arch set to this GPU's."""
    src = os.path.join(REF_CODE, "backend_cuda.cu")
    harness = os.path.join(HERE, "ref_gpu_harness.cpp")
    hdrs = [os.path.join(REF_CODE, f) for f in ("backend.hpp", "barnett.hpp", "kroupa.hpp")]
    if not os.path.exists(src) or not os.path.exists(NVCC):
        return
    if force or _stale(REF_CUDA_SO, [src, harness, *hdrs, __file__]):
        _run([NVCC, "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++14", "-DWITH_CUDA",
              "-Xcompiler", "-fPIC,-O3,-march=x86-64-v3", "-shared", "-I", REF_CODE,
              "-I", os.path.join(REPO, "include"), src, harness, "-o", REF_CUDA_SO])


if __name__ == "__main__":
    # python oracle/build_oracle.py [--force] [<reference>/Code]
    refs = [a for a in sys.argv[1:] if not a.startswith("--")]
    build(force="--force" in sys.argv, reference=refs[0] if refs else None)
