"""Python host API of the B200 displacement backend.

It mirrors the reference's backend interface (Code/backend.hpp): LoopData,
AtomArrays, BackendTiming, GpuOptions, gpu_available, print_gpu_info,
gpu_line_fp64 and kroupa_gpu keep the reference's names, argument meanings and
accumulate-into-u semantics, and every call goes through the C-ABI of
libdisco_b200.so.  Plan is the resident form: loop tables uploaded once,
atoms already on the device.
"""
from dataclasses import dataclass, field
import ctypes

import numpy as np

from . import _capi as C


@dataclass
class LoopPhys:
    """Code/kroupa.hpp:28-36: b = |b| per axis, unit m and n, loopon area dS."""
    bx: float = 0.0
    by: float = 0.0
    bz: float = 0.0
    mx: float = 0.0
    my: float = 0.0
    mz: float = 0.0
    nx: float = 0.0
    ny: float = 0.0
    nz: float = 0.0
    dS: float = 0.0

    def as_c(self):
        return C.DiscoLoopPhys(self.bx, self.by, self.bz, self.mx, self.my, self.mz,
                               self.nx, self.ny, self.nz, self.dS)


@dataclass
class LoopData:
    """Code/backend.hpp:20-26: loopons x/y/z, physics, line flag, polyline, apex."""
    x: np.ndarray = field(default_factory=lambda: np.zeros(0))
    y: np.ndarray = field(default_factory=lambda: np.zeros(0))
    z: np.ndarray = field(default_factory=lambda: np.zeros(0))
    phys: LoopPhys = field(default_factory=LoopPhys)
    line: bool = False
    vx: np.ndarray = field(default_factory=lambda: np.zeros(0))
    vy: np.ndarray = field(default_factory=lambda: np.zeros(0))
    vz: np.ndarray = field(default_factory=lambda: np.zeros(0))
    cx: float = 0.0
    cy: float = 0.0
    cz: float = 0.0

    def burgers(self):
        """b = (|b|_x m_x, |b|_y m_y, |b|_z m_z) (Code/backend_cpu.cpp:44-45)."""
        p = self.phys
        return np.array([p.bx * p.mx, p.by * p.my, p.bz * p.mz])


@dataclass
class AtomArrays:
    """Code/backend.hpp:29-33: positions read, displacements accumulated."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    ux: np.ndarray
    uy: np.ndarray
    uz: np.ndarray

    @property
    def n(self):
        return int(self.x.shape[0])

    @staticmethod
    def zeros_like_positions(x, y, z):
        n = len(x)
        return AtomArrays(np.ascontiguousarray(x, dtype=np.float64),
                          np.ascontiguousarray(y, dtype=np.float64),
                          np.ascontiguousarray(z, dtype=np.float64),
                          np.zeros(n), np.zeros(n), np.zeros(n))


@dataclass
class BackendTiming:
    """Code/backend.hpp:36-39 (seconds)."""
    upload: float = 0.0
    kernels: float = 0.0
    download: float = 0.0
    loopSec: list = field(default_factory=list)


@dataclass
class GpuOptions:
    """Code/backend.hpp:53-56."""
    fp32: bool = False
    chunkPairs: float = -1.0


def _f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a


def loop_array(loops):
    """ctypes array of DiscoLoop for `loops` plus the numpy buffers it points to."""
    keep = []
    arr = (C.DiscoLoop * max(1, len(loops)))()
    for i, lp in enumerate(loops):
        d = arr[i]
        xs = [_f64(lp.x), _f64(lp.y), _f64(lp.z)]
        vs = [_f64(lp.vx), _f64(lp.vy), _f64(lp.vz)]
        keep += xs + vs
        d.x, d.y, d.z = (a.ctypes.data if a.size else None for a in xs)
        d.n_loopons = int(xs[0].shape[0])
        d.line = 1 if lp.line else 0
        d.phys = lp.phys.as_c()
        d.vx, d.vy, d.vz = (a.ctypes.data if a.size else None for a in vs)
        d.n_vertices = int(vs[0].shape[0])
        d.cx, d.cy, d.cz = float(lp.cx), float(lp.cy), float(lp.cz)
    return arr, keep


def options(precision=C.DISCO_FP64, images=1, nu=0.35, image_split=0, verbose=0, near_plane=0.0,
            near_rim=0.0, image_min=0):
    lib = C.cuda_lib()
    o = C.DiscoOptions()
    lib.disco_b200_options_default(ctypes.byref(o))
    o.precision = precision
    o.images = images
    o.nu = nu
    o.image_split = image_split
    o.verbose = verbose
    o.near_plane = near_plane
    o.near_rim = near_rim
    o.image_min = image_min
    return o


def gpu_available():
    """Code/backend.hpp:58 gpuAvailable()."""
    return bool(C.cuda_lib().disco_b200_available())


def gpu_info():
    buf = ctypes.create_string_buffer(512)
    lib = C.cuda_lib()
    C.check(lib.disco_b200_device_info(buf, 512), lib)
    return buf.value.decode()


def print_gpu_info():
    """Code/backend.hpp:59 printGpuInfo()."""
    print(gpu_info(), end="")


def gpu_line_fp64():
    """Code/backend.hpp:60 gpuLineFp64()."""
    return bool(C.cuda_lib().disco_b200_line_fp64())


def kroupa_gpu(atoms, loops, dx, dy, dz, opt=None, t=None, *, images=1, nu=0.35, image_split=0,
               verbose=0, near_plane=0.0, near_rim=0.0, image_min=0):
    """kroupaGPU (Code/backend.hpp:61-62): adds the field of every loop over its
    periodic images into atoms.ux/uy/uz.  images and nu default to the
    reference's fixed values (+-1, 0.35).  Raises DiscoError on failure."""
    opt = opt or GpuOptions()
    lib = C.cuda_lib()
    o = options(C.DISCO_FP32C if opt.fp32 else C.DISCO_FP64, images, nu, image_split, verbose,
                near_plane, near_rim, image_min)
    o.chunk_pairs = opt.chunkPairs
    for name in ("x", "y", "z", "ux", "uy", "uz"):
        a = getattr(atoms, name)
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError(f"atoms.{name} must be a contiguous float64 array")
    a = C.DiscoAtoms(atoms.x.ctypes.data, atoms.y.ctypes.data, atoms.z.ctypes.data,
                     atoms.ux.ctypes.data, atoms.uy.ctypes.data, atoms.uz.ctypes.data, atoms.n)
    arr, keep = loop_array(loops)
    loop_sec = np.zeros(max(1, len(loops)))
    tm = C.DiscoTiming(0.0, 0.0, 0.0, loop_sec.ctypes.data)
    box = (ctypes.c_double * 3)(dx, dy, dz)
    C.check(lib.disco_b200_displace(ctypes.byref(a), arr, len(loops), box, ctypes.byref(o),
                                    ctypes.byref(tm)), lib)
    if t is not None:
        t.upload, t.kernels, t.download = tm.upload, tm.kernels, tm.download
        t.loopSec = list(loop_sec[:len(loops)])
    del keep
    return atoms


class Plan:
    """Resident form: loop tables built and uploaded once; execute() adds the
    field into device arrays (torch tensors or raw device pointers)."""

    def __init__(self, loops, box, *, precision=C.DISCO_FP64, images=1, nu=0.35, image_split=0,
                 max_atoms=0, image_min=0, near_plane=0.0, near_rim=0.0):
        self._lib = C.cuda_lib()
        o = options(precision, images, nu, image_split, image_min=image_min, near_plane=near_plane,
                    near_rim=near_rim)
        arr, keep = loop_array(loops)
        b = (ctypes.c_double * 3)(*[float(v) for v in box])
        h = ctypes.c_void_p()
        C.check(self._lib.disco_b200_plan_create(arr, len(loops), b, ctypes.byref(o), max_atoms,
                                                 ctypes.byref(h)), self._lib)
        self._h = h
        del keep

    def stats(self):
        s = C.DiscoPlanStats()
        C.check(self._lib.disco_b200_plan_stats(self._h, ctypes.byref(s)), self._lib)
        return {k: getattr(s, k) for k, _ in C.DiscoPlanStats._fields_}

    def execute_ptrs(self, x, y, z, ux, uy, uz, n, stream=0):
        a = C.DiscoAtoms(x, y, z, ux, uy, uz, n)
        C.check(self._lib.disco_b200_plan_execute(self._h, ctypes.byref(a), ctypes.c_void_p(stream)),
                self._lib)

    def execute(self, pos, u, stream=None):
        """pos, u: (3, n) float64 CUDA tensors (rows x, y, z).  Adds into u."""
        import torch
        assert pos.dtype == torch.float64 and u.dtype == torch.float64
        assert pos.is_cuda and u.is_cuda and pos.is_contiguous() and u.is_contiguous()
        n = pos.shape[1]
        s = (stream or torch.cuda.current_stream()).cuda_stream
        self.execute_ptrs(pos[0].data_ptr(), pos[1].data_ptr(), pos[2].data_ptr(),
                          u[0].data_ptr(), u[1].data_ptr(), u[2].data_ptr(), n, s)

    def sync(self, stream=0):
        C.check(self._lib.disco_b200_plan_sync(self._h, ctypes.c_void_p(stream)), self._lib)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.disco_b200_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sample_array(workloads, us=None, device_ptrs=None):
    """ctypes DiscoSample array for a batch (host arrays, or device pointers
    given as [(x, y, z, ux, uy, uz), ...])."""
    keep = []
    arr = (C.DiscoSample * max(1, len(workloads)))()
    for i, w in enumerate(workloads):
        la, lk = loop_array(w.loops)
        keep += [la, lk]
        d = arr[i]
        if device_ptrs is not None:
            d.atoms = C.DiscoAtoms(*device_ptrs[i], w.n)
        else:
            u = us[i]
            xs = [_f64(w.x), _f64(w.y), _f64(w.z)]
            keep += xs
            d.atoms = C.DiscoAtoms(xs[0].ctypes.data, xs[1].ctypes.data, xs[2].ctypes.data,
                                   u[0].ctypes.data, u[1].ctypes.data, u[2].ctypes.data, w.n)
        d.loops = ctypes.cast(la, ctypes.c_void_p)
        d.nloops = len(w.loops)
        d.images = w.images
        d.box = C.D3(*w.box)
        d.image_min = getattr(w, "image_min", 0)
    return arr, keep


def batch_gpu(workloads, precision=C.DISCO_FP64, nu=None, image_split=0, stage_kb=0, stages=0,
              near_plane=0.0, near_rim=0.0):
    """The batched form on host arrays: returns [(ux, uy, uz)] per sample."""
    lib = C.cuda_lib()
    nu = workloads[0].nu if nu is None else nu
    us = [[np.zeros(w.n), np.zeros(w.n), np.zeros(w.n)] for w in workloads]
    arr, keep = sample_array(workloads, us)
    o = options(precision, 1, nu, image_split, near_plane=near_plane, near_rim=near_rim)
    o.stage_kb = stage_kb
    o.stages = stages
    tm = C.DiscoTiming(0.0, 0.0, 0.0, None)
    C.check(lib.disco_b200_batch(arr, len(workloads), ctypes.byref(o), ctypes.byref(tm)), lib)
    del keep
    return us, tm.kernels


class BatchPlan:
    """Resident batched form: tables, unit queue and CUDA graph built once;
    atoms are device arrays given as [(x, y, z, ux, uy, uz) pointers]."""

    def __init__(self, workloads, device_ptrs, *, precision=C.DISCO_FP64, nu=None, image_split=0,
                 stage_kb=0, stages=0):
        self._lib = C.cuda_lib()
        nu = workloads[0].nu if nu is None else nu
        arr, keep = sample_array(workloads, device_ptrs=device_ptrs)
        o = options(precision, 1, nu, image_split)
        o.stage_kb = stage_kb
        o.stages = stages
        h = ctypes.c_void_p()
        C.check(self._lib.disco_b200_batch_plan_create(arr, len(workloads), ctypes.byref(o),
                                                       ctypes.byref(h)), self._lib)
        self._h = h
        del keep

    def execute(self, stream=0):
        C.check(self._lib.disco_b200_batch_plan_execute(self._h, ctypes.c_void_p(stream)), self._lib)

    def sync(self, stream=0):
        C.check(self._lib.disco_b200_batch_plan_sync(self._h, ctypes.c_void_p(stream)), self._lib)

    def stats(self):
        s = C.DiscoPlanStats()
        C.check(self._lib.disco_b200_batch_plan_stats(self._h, ctypes.byref(s)), self._lib)
        return {k: getattr(s, k) for k, _ in C.DiscoPlanStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.disco_b200_batch_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
