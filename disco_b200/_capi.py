"""ctypes mirror of include/disco_b200.h and include/disco_geometry.h.

The structures below are field-for-field the C structures; the libraries are
loaded from disco_b200/_lib.  A missing library raises at import time: there
is no fallback path.
"""
import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_int, c_int8, c_int32, c_int64,
                    c_size_t, c_void_p)

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib")
CUDA_LIB_PATH = os.path.join(LIB_DIR, "libdisco_b200.so")
GEOM_LIB_PATH = os.path.join(LIB_DIR, "libdisco_geom.so")
SHIM_LIB_PATH = os.path.join(LIB_DIR, "libdisco_backend.so")

DISCO_OK, DISCO_EINVAL, DISCO_ENODEV, DISCO_ECUDA = 0, 1, 2, 3
DISCO_ENOMEM, DISCO_ELIMIT, DISCO_ETIMEOUT, DISCO_EPLANES = 4, 5, 6, 7
DISCO_FP64, DISCO_FP32C = 0, 1
SHAPE_CIRCLE, SHAPE_RECTANGLE, SHAPE_PARALLELOGRAM, SHAPE_POLYGON = 0, 1, 2, 3
MAX_POLY = 32
MATTER_NONE, MATTER_VACANCY, MATTER_INTERSTITIAL = 0, 1, 2
LATTICE_BCC, LATTICE_FCC = 0, 1

D3 = c_double * 3
DP = c_double * MAX_POLY


class DiscoAtoms(Structure):
    _fields_ = [("x", c_void_p), ("y", c_void_p), ("z", c_void_p),
                ("ux", c_void_p), ("uy", c_void_p), ("uz", c_void_p), ("n", c_int64)]


class DiscoLoopPhys(Structure):
    _fields_ = [(k, c_double) for k in ("bx", "by", "bz", "mx", "my", "mz", "nx", "ny", "nz", "dS")]


class DiscoLoop(Structure):
    _fields_ = [("x", c_void_p), ("y", c_void_p), ("z", c_void_p),
                ("n_loopons", c_int32), ("line", c_int32), ("phys", DiscoLoopPhys),
                ("vx", c_void_p), ("vy", c_void_p), ("vz", c_void_p),
                ("n_vertices", c_int32), ("reserved", c_int32),
                ("cx", c_double), ("cy", c_double), ("cz", c_double)]


class DiscoOptions(Structure):
    _fields_ = [("precision", c_int32), ("images", c_int32), ("nu", c_double),
                ("chunk_pairs", c_double), ("atoms_per_thread", c_int32),
                ("threads_per_block", c_int32), ("image_split", c_int32), ("verbose", c_int32),
                ("near_plane", c_double), ("near_rim", c_double), ("stage_kb", c_int32),
                ("image_min", c_int32), ("stages", c_int32), ("reserved", c_int32)]


class DiscoSample(Structure):
    _fields_ = [("atoms", DiscoAtoms), ("loops", c_void_p), ("nloops", c_int32), ("images", c_int32),
                ("box", D3), ("image_min", c_int32), ("reserved", c_int32)]


class DiscoTiming(Structure):
    _fields_ = [("upload", c_double), ("kernels", c_double), ("download", c_double),
                ("loop_sec", c_void_p)]


class DiscoPlanStats(Structure):
    _fields_ = [("n_loops", c_int64), ("n_line_loops", c_int64), ("n_loopon_loops", c_int64),
                ("n_segments", c_int64), ("n_loopons", c_int64), ("n_images", c_int64),
                ("evals_per_atom", c_double)]


class DiscoSlabLoop(Structure):
    _fields_ = [("c", D3), ("m", D3), ("n", D3), ("bmag", c_double), ("u", D3), ("v", D3),
                ("spacing", c_double), ("shape", c_int32), ("n_poly", c_int32),
                ("radius", c_double), ("half_m", c_double), ("half_p", c_double),
                ("r_corner", c_double),
                ("pu", DP), ("pv", DP), ("qu", DP), ("qv", DP), ("nu", DP), ("nv", DP),
                ("shift_pos", D3), ("shift_neg", D3), ("apply", c_int32), ("reserved", c_int32)]


class DiscoSlabInfo(Structure):
    _fields_ = [("type", c_int32), ("planes", c_int32), ("height", c_double),
                ("spacing", c_double), ("b", D3), ("offset", c_int64), ("count", c_int64)]


class DiscoCopy(Structure):
    _fields_ = [("atom", c_int32), ("reserved", c_int32), ("shift", D3)]


class DiscoGeomLoop(Structure):
    _fields_ = [("shape", c_int32), ("n_poly", c_int32), ("c", D3), ("m", D3), ("n", D3),
                ("p", D3), ("u", D3), ("v", D3), ("bmag", c_double), ("radius", c_double),
                ("half_m", c_double), ("half_p", c_double), ("r_corner", c_double),
                ("da", c_double), ("dS", c_double),
                ("pu", DP), ("pv", DP), ("qu", DP), ("qv", DP), ("nu", DP), ("nv", DP)]


class DiscoFarNorm(Structure):
    _fields_ = [("mu", ctypes.c_float * 16), ("inv_sd", ctypes.c_float * 16), ("out_scale", ctypes.c_float),
                ("images", c_int32), ("image_min", c_int32), ("reserved", c_int32)]


class DiscoLearnedOptions(Structure):
    _fields_ = [("precision", c_int32), ("check_precision", c_int32), ("nu", c_double),
                ("check_fraction", c_double), ("tol_loop", c_double), ("tol_total", c_double),
                ("seed", ctypes.c_uint64)]


class DiscoLearnedReport(Structure):
    _fields_ = [("n_check", c_int64), ("n_fallback", c_int32), ("launches", c_int32),
                ("check_max", c_double), ("check_rms", c_double), ("worst_loop", c_double),
                ("t_check", c_double), ("t_near", c_double), ("t_far", c_double), ("t_fallback", c_double),
                ("loop_err", c_void_p), ("fallback", c_void_p)]


class DiscoError(RuntimeError):
    """A non-zero status of a C-ABI call; .status holds the code."""

    def __init__(self, status, message):
        super().__init__(f"status {status}: {message}")
        self.status = status


def _load(path, what):
    if not os.path.exists(path):
        raise ImportError(f"{what} not built: {path} is missing (run __graft_entry__.build())")
    return ctypes.CDLL(path)


def _sig(lib, name, restype, argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = argtypes
    return f


_cuda = None
_geom = None


def cuda_lib():
    """libdisco_b200.so with its prototypes set (loaded once)."""
    global _cuda
    if _cuda is None:
        lib = _load(CUDA_LIB_PATH, "CUDA backend library")
        _sig(lib, "disco_b200_available", c_int, [])
        _sig(lib, "disco_b200_device_info", c_int, [c_char_p, c_size_t])
        _sig(lib, "disco_b200_line_fp64", c_int, [])
        _sig(lib, "disco_b200_options_default", None, [POINTER(DiscoOptions)])
        _sig(lib, "disco_b200_last_error", c_char_p, [])
        _sig(lib, "disco_b200_strerror", c_char_p, [c_int])
        _sig(lib, "disco_b200_displace", c_int,
             [POINTER(DiscoAtoms), POINTER(DiscoLoop), c_int32, POINTER(c_double),
              POINTER(DiscoOptions), POINTER(DiscoTiming)])
        _sig(lib, "disco_b200_plan_create", c_int,
             [POINTER(DiscoLoop), c_int32, POINTER(c_double), POINTER(DiscoOptions), c_int64,
              POINTER(c_void_p)])
        _sig(lib, "disco_b200_plan_execute", c_int, [c_void_p, POINTER(DiscoAtoms), c_void_p])
        _sig(lib, "disco_b200_plan_sync", c_int, [c_void_p, c_void_p])
        _sig(lib, "disco_b200_plan_stats", c_int, [c_void_p, POINTER(DiscoPlanStats)])
        _sig(lib, "disco_b200_plan_destroy", c_int, [c_void_p])
        _sig(lib, "disco_b200_batch", c_int,
             [POINTER(DiscoSample), c_int32, POINTER(DiscoOptions), POINTER(DiscoTiming)])
        _sig(lib, "disco_b200_batch_plan_create", c_int,
             [POINTER(DiscoSample), c_int32, POINTER(DiscoOptions), POINTER(c_void_p)])
        _sig(lib, "disco_b200_batch_plan_execute", c_int, [c_void_p, c_void_p])
        _sig(lib, "disco_b200_batch_plan_sync", c_int, [c_void_p, c_void_p])
        _sig(lib, "disco_b200_batch_plan_stats", c_int, [c_void_p, POINTER(DiscoPlanStats)])
        _sig(lib, "disco_b200_batch_plan_destroy", c_int, [c_void_p])
        _sig(lib, "disco_b200_mlp_create", c_int, [ctypes.c_uint64, POINTER(c_void_p)])
        _sig(lib, "disco_b200_mlp_destroy", c_int, [c_void_p])
        _sig(lib, "disco_b200_mlp_param_count", c_int, [])
        _sig(lib, "disco_b200_mlp_get_params", c_int, [c_void_p, c_void_p])
        _sig(lib, "disco_b200_mlp_set_params", c_int, [c_void_p, c_void_p])
        _sig(lib, "disco_b200_mlp_get_grads", c_int, [c_void_p, c_void_p])
        _sig(lib, "disco_b200_mlp_forward", c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p])
        _sig(lib, "disco_b200_mlp_grad", c_int,
             [c_void_p, c_void_p, c_void_p, c_int64, POINTER(ctypes.c_float), c_void_p])
        _sig(lib, "disco_b200_mlp_adam", c_int,
             [c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
              c_void_p])
        _sig(lib, "disco_b200_mlp_status", c_int, [c_void_p])
        _sig(lib, "disco_b200_format_atoms", c_int,
             [c_int32, c_char_p, c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_int64, POINTER(c_int64),
              c_void_p])
        _sig(lib, "disco_b200_lattice", c_int,
             [c_int32, c_int32, c_int32, c_int32, c_double, c_void_p, c_void_p, c_void_p, c_void_p])
        _sig(lib, "disco_b200_math_check", c_int, [c_int32, c_void_p, c_void_p, c_int64, c_void_p])
        _sig(lib, "disco_b200_far_features", c_int,
             [POINTER(DiscoAtoms), POINTER(DiscoLoop), c_int32, POINTER(c_double), POINTER(DiscoFarNorm),
              c_void_p, c_void_p, c_void_p])
        _sig(lib, "disco_b200_far_apply", c_int,
             [c_void_p, POINTER(DiscoFarNorm), POINTER(DiscoAtoms), POINTER(DiscoLoop), c_int32,
              POINTER(c_double), c_void_p, c_int32, c_void_p, c_void_p])
        _sig(lib, "disco_b200_learned_displace", c_int,
             [c_void_p, POINTER(DiscoFarNorm), POINTER(DiscoAtoms), POINTER(DiscoLoop), c_int32,
              POINTER(c_double), POINTER(DiscoLearnedOptions), POINTER(DiscoLearnedReport), c_void_p])
        _sig(lib, "disco_b200_prismatic", c_int,
             [c_void_p, c_void_p, c_void_p, c_int64, POINTER(DiscoSlabLoop), c_int32,
              POINTER(c_double), c_void_p, c_void_p, c_void_p, c_void_p, POINTER(DiscoSlabInfo),
              c_void_p, c_void_p, c_int64, POINTER(DiscoCopy), c_int64, POINTER(c_int64)])
        _sig(lib, "disco_b200_prismatic_noalloc", c_int,
             [c_void_p, c_void_p, c_void_p, c_int64, POINTER(DiscoSlabLoop), c_int32,
              POINTER(c_double), c_void_p, c_void_p, c_void_p, c_void_p, POINTER(DiscoSlabInfo),
              c_void_p, c_void_p, c_int64, c_void_p, c_int64, POINTER(c_int64), c_void_p])
        _sig(lib, "disco_b200_finalize", c_int,
             [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
              POINTER(DiscoCopy), c_int64, POINTER(c_double), c_void_p, c_void_p, c_void_p,
              c_void_p, c_void_p, c_void_p])
        _sig(lib, "disco_b200_finalize_resident", c_int,
             [c_void_p] * 6 + [c_int64, c_void_p, c_int64, POINTER(c_double)] + [c_void_p] * 7)
        _cuda = lib
    return _cuda


def geom_lib():
    """libdisco_geom.so with its prototypes set (loaded once)."""
    global _geom
    if _geom is None:
        lib = _load(GEOM_LIB_PATH, "geometry library")
        GP = POINTER(DiscoGeomLoop)
        DPTR = POINTER(c_double)
        _sig(lib, "disco_geom_circle", c_int, [c_double, c_double, DPTR, DPTR, DPTR, c_double, GP])
        _sig(lib, "disco_geom_rectangle", c_int,
             [c_double, c_double, c_double, c_double, DPTR, DPTR, DPTR, c_double, DPTR, GP])
        _sig(lib, "disco_geom_parallelogram", c_int,
             [c_double, c_double, c_double, DPTR, DPTR, DPTR, DPTR, DPTR, c_double, GP])
        _sig(lib, "disco_geom_polygon", c_int,
             [c_double, DPTR, c_int32, c_double, DPTR, DPTR, DPTR, c_double, DPTR, GP])
        _sig(lib, "disco_geom_regular_polygon", c_int, [c_int32, c_double, DPTR, DPTR, DPTR, DPTR])
        _sig(lib, "disco_geom_polyline", c_int32, [GP, c_double, DPTR, c_int32])
        _sig(lib, "disco_geom_loopons", c_int64, [GP, DPTR, c_int64])
        _sig(lib, "disco_geom_area", c_double, [GP])
        _sig(lib, "disco_geom_contains", c_int, [GP, DPTR])
        _sig(lib, "disco_geom_snap", c_int,
             [DPTR, DPTR, c_double, c_int32, c_int32, c_int32, c_int32, DPTR, DPTR])
        _sig(lib, "disco_geom_lattice", c_int64,
             [c_int32, c_int32, c_int32, c_int32, c_double, c_void_p, c_void_p, c_void_p])
        _sig(lib, "disco_geom_classify_burgers", c_int32, [c_int32, DPTR, DPTR])
        _sig(lib, "disco_geom_slab_loop", c_int,
             [GP, c_double, c_int32, c_int32, c_double, POINTER(DiscoSlabLoop)])
        _geom = lib
    return _geom


def check(status, lib=None):
    """Raises DiscoError for a non-zero status, with the library's message."""
    if status != DISCO_OK:
        msg = ""
        lib = lib or _cuda
        if lib is not None and hasattr(lib, "disco_b200_last_error"):
            msg = (lib.disco_b200_last_error() or b"").decode()
        raise DiscoError(status, msg or "error")
    return status


def d3(v):
    return D3(*[float(t) for t in v])
