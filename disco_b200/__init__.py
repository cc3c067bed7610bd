"""disco_b200 — B200-native (sm_100a) displacement backend for DISCO.

The hot path of DISCO (the per-atom elastic field of every dislocation loop
over its periodic images, Barnett line integral or Kroupa loopons, plus the
prismatic slab selection and compaction) as hand-written CUDA kernels behind a
C-ABI (include/disco_b200.h).  The Python modules call that C-ABI through
ctypes: backend (the reference's backend interface), geometry (input
synthesis), workloads (seeded synthetic inputs), prismatic (matter step).
"""
from .backend import (AtomArrays, BackendTiming, GpuOptions, LoopData, LoopPhys, Plan,  # noqa: F401
                      gpu_available, gpu_info, gpu_line_fp64, kroupa_gpu, print_gpu_info)
from ._capi import DiscoError, DISCO_FP64, DISCO_FP32C  # noqa: F401
