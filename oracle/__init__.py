"""ORACLE — test infrastructure only (the checker, never the product path).

ctypes access to the CPU restatement (oracle/_build/libdisco_oracle*.so, from
oracle/disco_oracle.cpp) and to the reference's own code compiled in place
(oracle/_ref/libdisco_ref.so, from oracle/ref_harness.cpp).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this package.
"""
import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_int32, c_int64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libdisco_oracle.so")
ORACLE_NOFMA_SO = os.path.join(HERE, "_build", "libdisco_oracle_nofma.so")
REF_SO = os.path.join(HERE, "_ref", "libdisco_ref.so")
REF_NOFMA_SO = os.path.join(HERE, "_ref", "libdisco_ref_nofma.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libdisco_ref_cuda.so")

_libs = {}


def _capi():
    from disco_b200 import _capi as C
    return C


def _load(path):
    if path not in _libs:
        if not os.path.exists(path):
            raise ImportError(f"oracle library missing: {path} (run oracle/build_oracle.py)")
        lib = ctypes.CDLL(path)
        C = _capi()
        if "libdisco_ref_cuda" in path:
            lib.ref_gpu_available.restype = c_int
            lib.ref_kroupa_gpu.restype = c_int
            lib.ref_kroupa_gpu.argtypes = [POINTER(C.DiscoAtoms), POINTER(C.DiscoLoop), c_int,
                                           POINTER(c_double), c_int, c_void_p]
        elif "libdisco_ref" in path:
            lib.ref_kroupa_cpu.restype = c_int
            lib.ref_kroupa_cpu.argtypes = [POINTER(C.DiscoAtoms), POINTER(C.DiscoLoop), c_int,
                                           POINTER(c_double), c_void_p]
            lib.ref_loop_new.restype = c_void_p
            lib.ref_loop_new.argtypes = [c_int, c_double, c_double, c_double, c_double, c_double,
                                         c_void_p, c_void_p, c_void_p, c_double, c_void_p, c_void_p,
                                         c_int, c_void_p, c_void_p]
            lib.ref_loop_free.argtypes = [c_void_p]
            lib.ref_loop_polyline.restype = c_int
            lib.ref_loop_polyline.argtypes = [c_void_p, c_double, c_void_p, c_int]
            lib.ref_loop_loopons.restype = c_int
            lib.ref_loop_loopons.argtypes = [c_void_p, c_void_p, c_int, POINTER(c_double)]
            lib.ref_loop_info.argtypes = [c_void_p, c_void_p]
            lib.ref_loop_contains.restype = c_int
            lib.ref_loop_contains.argtypes = [c_void_p, c_void_p]
            lib.ref_snap.argtypes = [c_void_p, c_void_p, c_double, c_int, c_int, c_int, c_int,
                                     c_void_p, POINTER(c_double)]
            lib.ref_regular_polygon.argtypes = [c_int, c_double, c_void_p, c_void_p, c_void_p, c_void_p]
            lib.ref_lattice.restype = c_int64
            lib.ref_lattice.argtypes = [c_int, c_int, c_int, c_int, c_double, c_void_p, c_void_p, c_void_p]
            lib.ref_prismatic_step.restype = c_int
            lib.ref_prismatic_step.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_int,
                                               c_void_p, c_void_p, c_void_p, c_int64, POINTER(c_double),
                                               c_void_p, c_void_p, c_void_p, c_void_p,
                                               POINTER(C.DiscoSlabInfo), c_void_p, c_void_p, c_int64,
                                               POINTER(C.DiscoCopy), c_int64, POINTER(c_int64)]
            lib.ref_classify_burgers.restype = c_int
            lib.ref_classify_burgers.argtypes = [c_int, c_void_p, c_void_p]
            lib.ref_threads.restype = c_int
            lib.ref_barnett_loop.argtypes = [c_double] * 3 + [c_void_p] * 3 + [c_int] + \
                [c_double] * 6 + [c_void_p]
            lib.ref_kroupa_pair.argtypes = [c_double] * 3 + [POINTER(C.DiscoLoopPhys), c_void_p]
        else:
            lib.oracle_threads.restype = c_int
            lib.oracle_barnett_loop.argtypes = [c_double, c_double, c_double, c_void_p, c_void_p,
                                                c_void_p, c_int, c_double, c_double, c_double,
                                                c_double, c_double, c_double, c_double, c_void_p]
            lib.oracle_kroupa_pair.argtypes = [c_double, c_double, c_double, POINTER(C.DiscoLoopPhys),
                                               c_double, c_void_p]
            lib.oracle_displace.restype = c_int
            lib.oracle_displace.argtypes = [POINTER(C.DiscoAtoms), POINTER(C.DiscoLoop), c_int,
                                            POINTER(c_double), c_int, c_double, c_int, c_void_p]
            lib.oracle_displace_shells.restype = c_int
            lib.oracle_displace_shells.argtypes = [POINTER(C.DiscoAtoms), POINTER(C.DiscoLoop), c_int,
                                                   POINTER(c_double), c_int, c_int, c_double, c_int,
                                                   c_void_p]
            lib.oracle_format_atoms.restype = c_int64
            lib.oracle_format_atoms.argtypes = [c_int, ctypes.c_char_p, c_void_p, c_void_p, c_void_p, c_int64,
                                                c_void_p, c_int64]
            lib.oracle_prismatic.restype = c_int
            lib.oracle_prismatic.argtypes = [c_void_p, c_void_p, c_void_p, c_int64,
                                             POINTER(C.DiscoSlabLoop), c_int32, POINTER(c_double),
                                             c_void_p, c_void_p, c_void_p, c_void_p,
                                             POINTER(C.DiscoSlabInfo), c_void_p, c_void_p, c_int64,
                                             POINTER(C.DiscoCopy), c_int64, POINTER(c_int64)]
            lib.oracle_finalize.restype = c_int
            lib.oracle_finalize.argtypes = [c_void_p] * 6 + [c_int64, POINTER(C.DiscoCopy), c_int64,
                                                              POINTER(c_double)] + [c_void_p] * 6
            lib.oracle_slab_margins.restype = c_int
            lib.oracle_slab_margins.argtypes = [c_void_p, c_void_p, c_void_p, c_int64,
                                                POINTER(C.DiscoSlabLoop), c_int32, POINTER(c_double),
                                                c_void_p]
        _libs[path] = lib
    return _libs[path]


def oracle_lib(nofma=False):
    return _load(ORACLE_NOFMA_SO if nofma else ORACLE_SO)


def ref_lib(nofma=False):
    return _load(REF_NOFMA_SO if nofma else REF_SO)


def have_ref():
    return os.path.exists(REF_SO)


def have_ref_cuda():
    return os.path.exists(REF_CUDA_SO)


def _box(box):
    return (c_double * 3)(*[float(v) for v in box])


def _atoms(x, y, z):
    C = _capi()
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    u = [np.zeros(len(x)) for _ in range(3)]
    a = C.DiscoAtoms(x.ctypes.data, y.ctypes.data, z.ctypes.data,
                     u[0].ctypes.data, u[1].ctypes.data, u[2].ctypes.data, len(x))
    return a, (x, y, z), u


def displace(x, y, z, loops, box, images=1, nu=0.35, threads=0, nofma=False, loop_sec=None,
             image_min=0):
    """oracle_displace: (ux, uy, uz) of every loop over images -images..images
    (image_min > 0: only the shells image_min <= max|n| <= images)."""
    from disco_b200.backend import loop_array
    lib = oracle_lib(nofma)
    a, keep_x, u = _atoms(x, y, z)
    arr, keep = loop_array(loops)
    ls = np.zeros(max(1, len(loops)))
    st = lib.oracle_displace_shells(ctypes.byref(a), arr, len(loops), _box(box), images, image_min, nu,
                                    threads, ls.ctypes.data)
    assert st == 0
    if loop_sec is not None:
        loop_sec[:] = ls[:len(loops)]
    return u


def ref_displace(x, y, z, loops, box, loop_sec=None, nofma=False):
    """The reference's own kroupaCPU (images +-1, nu 0.35)."""
    from disco_b200.backend import loop_array
    lib = ref_lib(nofma)
    a, keep_x, u = _atoms(x, y, z)
    arr, keep = loop_array(loops)
    ls = np.zeros(max(1, len(loops)))
    st = lib.ref_kroupa_cpu(ctypes.byref(a), arr, len(loops), _box(box), ls.ctypes.data)
    assert st == 0
    if loop_sec is not None:
        loop_sec[:] = ls[:len(loops)]
    return u


def ref_displace_gpu(x, y, z, loops, box, fp32=False):
    """The reference's own kroupaGPU (Code/backend_cuda.cu, built for sm_100a;
    images +-1, nu 0.35): (ux, uy, uz) and its (upload, kernels, download)
    seconds as it measures them."""
    from disco_b200.backend import loop_array
    lib = _load(REF_CUDA_SO)
    a, keep_x, u = _atoms(x, y, z)
    arr, keep = loop_array(loops)
    t = np.zeros(3)
    st = lib.ref_kroupa_gpu(ctypes.byref(a), arr, len(loops), _box(box), int(fp32), t.ctypes.data)
    assert st == 0
    return u, t


def barnett_loop(p, V, c, b, nu):
    V = np.ascontiguousarray(V, dtype=np.float64)
    vx, vy, vz = (np.ascontiguousarray(V[:, k]) for k in range(3))
    out = np.zeros(3)
    oracle_lib().oracle_barnett_loop(float(p[0]), float(p[1]), float(p[2]), vx.ctypes.data,
                                     vy.ctypes.data, vz.ctypes.data, len(V), float(c[0]), float(c[1]),
                                     float(c[2]), float(b[0]), float(b[1]), float(b[2]), nu,
                                     out.ctypes.data)
    return out


def kroupa_pair(rho, phys, nu):
    out = np.zeros(3)
    oracle_lib().oracle_kroupa_pair(float(rho[0]), float(rho[1]), float(rho[2]),
                                    ctypes.byref(phys.as_c()), nu, out.ctypes.data)
    return out


def _prismatic_call(fn, x, y, z, slab_loops, box, extra=()):
    C = _capi()
    n = len(x)
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    nl = len(slab_loops)
    xo, yo, zo = np.empty(n), np.empty(n), np.empty(n)
    new_index = np.empty(n, dtype=np.int32)
    info = (C.DiscoSlabInfo * max(1, nl))()
    counts = (c_int64 * 3)()
    cap = 1 << 16
    while True:
        slab_atoms = np.empty(cap, dtype=np.int32)
        slab_side = np.empty(cap, dtype=np.int8)
        copies = (C.DiscoCopy * cap)()
        st = fn(*extra, x.ctypes.data, y.ctypes.data, z.ctypes.data, n, _box(box),
                xo.ctypes.data, yo.ctypes.data, zo.ctypes.data, new_index.ctypes.data, info,
                slab_atoms.ctypes.data, slab_side.ctypes.data, cap, copies, cap, counts)
        if st == C.DISCO_ELIMIT:
            cap = max(counts[1], counts[2]) + 16
            continue
        assert st == 0, st
        break
    k, ns, nc = counts[0], counts[1], counts[2]
    cp = np.array([(copies[i].atom, *copies[i].shift[:]) for i in range(nc)]).reshape(-1, 4)
    return {
        "survivors": (xo[:k].copy(), yo[:k].copy(), zo[:k].copy()),
        "new_index": new_index,
        "info": [(info[l].type, info[l].planes, info[l].height, info[l].spacing, tuple(info[l].b[:]),
                  info[l].offset, info[l].count) for l in range(nl)],
        "slab_atoms": slab_atoms[:ns].copy(),
        "slab_side": slab_side[:ns].copy(),
        "copy_atom": cp[:, 0].astype(np.int32) if nc else np.zeros(0, np.int32),
        "copy_shift": cp[:, 1:] if nc else np.zeros((0, 3)),
    }


def prismatic(x, y, z, slab_loops, box, nofma=True):
    """oracle_prismatic (pinned -ffp-contract=off build by default)."""
    C = _capi()
    lib = oracle_lib(nofma)
    nl = len(slab_loops)
    arr = (C.DiscoSlabLoop * max(1, nl))(*slab_loops)

    def fn(x_, y_, z_, n, box_, *rest):
        return lib.oracle_prismatic(x_, y_, z_, n, arr, nl, box_, *rest)
    return _prismatic_call(fn, x, y, z, slab_loops, box)


def slab_margins(x, y, z, slab_loops, box):
    C = _capi()
    lib = oracle_lib(True)
    nl = len(slab_loops)
    arr = (C.DiscoSlabLoop * max(1, nl))(*slab_loops)
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    out = np.zeros(2)
    lib.oracle_slab_margins(x.ctypes.data, y.ctypes.data, z.ctypes.data, len(x), arr, nl, _box(box),
                            out.ctypes.data)
    return out


def format_atoms(fmt, element, x, y, z):
    """oracle_format_atoms: the writers' atom lines as bytes (0 XYZ, 1 LAMMPS)."""
    lib = oracle_lib(False)
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    n = len(x)
    need = lib.oracle_format_atoms(fmt, element.encode(), x.ctypes.data, y.ctypes.data, z.ctypes.data, n, None, 0)
    buf = ctypes.create_string_buffer(max(1, need))
    lib.oracle_format_atoms(fmt, element.encode(), x.ctypes.data, y.ctypes.data, z.ctypes.data, n,
                            ctypes.addressof(buf), need)
    return buf.raw[:need]


def finalize(x, y, z, ux, uy, uz, copy_atom, copy_shift, box):
    C = _capi()
    lib = oracle_lib(True)
    n, nc = len(x), len(copy_atom)
    cps = (C.DiscoCopy * max(1, nc))()
    for i in range(nc):
        cps[i].atom = int(copy_atom[i])
        cps[i].shift = C.D3(*copy_shift[i])
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, ux, uy, uz)]
    out = [np.empty(n + nc) for _ in range(6)]
    st = lib.oracle_finalize(*[a.ctypes.data for a in arrs], n, cps, nc, _box(box),
                             *[o.ctypes.data for o in out])
    assert st == 0
    return out


# ---- the reference's own loop class and matter step ----------------------------------------

class RefLoop:
    """A reference `loop` object (Code/loop.hpp) built in oracle/_ref."""

    def __init__(self, shape, da, c, m, n, a0, radius=0.0, half_m=0.0, half_p=0.0, corner_r=0.0,
                 side=None, verts=None, dir1=None, dir2=None):
        lib = ref_lib()
        self._keep = []

        def arr(v):
            if v is None:
                return None
            a = np.ascontiguousarray(v, dtype=np.float64).ravel()
            self._keep.append(a)
            return a.ctypes.data
        nverts = 0 if verts is None else len(verts)
        self.h = lib.ref_loop_new(shape, da, radius, half_m, half_p, corner_r, arr(c), arr(m), arr(n),
                                  a0, arr(side), arr(verts), nverts, arr(dir1), arr(dir2))

    def polyline(self, eps):
        lib = ref_lib()
        n = lib.ref_loop_polyline(self.h, eps, None, 0)
        out = np.empty((n, 3))
        lib.ref_loop_polyline(self.h, eps, out.ctypes.data, n)
        return out

    def loopons(self):
        lib = ref_lib()
        dS = c_double()
        n = lib.ref_loop_loopons(self.h, None, 0, ctypes.byref(dS))
        out = np.empty((n, 3))
        lib.ref_loop_loopons(self.h, out.ctypes.data, n, ctypes.byref(dS))
        return out, dS.value

    def info(self):
        out = np.zeros(14)
        ref_lib().ref_loop_info(self.h, out.ctypes.data)
        return {"c": out[0:3], "m": out[3:6], "n": out[6:9], "b": out[9:12], "area": out[12],
                "r_corner": out[13]}

    def contains(self, rel):
        r = np.ascontiguousarray(rel, dtype=np.float64)
        return bool(ref_lib().ref_loop_contains(self.h, r.ctypes.data))

    def __del__(self):
        try:
            ref_lib().ref_loop_free(self.h)
        except Exception:
            pass


def ref_snap(c, n, a0, nx, ny, nz, lattice):
    out = np.zeros(3)
    d = c_double()
    c = np.ascontiguousarray(c, dtype=np.float64)
    n = np.ascontiguousarray(n, dtype=np.float64)
    ref_lib().ref_snap(c.ctypes.data, n.ctypes.data, a0, nx, ny, nz, lattice, out.ctypes.data,
                       ctypes.byref(d))
    return out, d.value


def ref_regular_polygon(sides, R, m, n, vertex_dir=None):
    out = np.empty((sides, 3))
    m = np.ascontiguousarray(m, dtype=np.float64)
    n = np.ascontiguousarray(n, dtype=np.float64)
    vd = None if vertex_dir is None else np.ascontiguousarray(vertex_dir, dtype=np.float64)
    ref_lib().ref_regular_polygon(sides, R, None if vd is None else vd.ctypes.data, m.ctypes.data,
                                  n.ctypes.data, out.ctypes.data)
    return out


def ref_lattice(lattice, nx, ny, nz, a0):
    nb = 4 if lattice == 1 else 2
    n = nb * nx * ny * nz
    x, y, z = np.empty(n), np.empty(n), np.empty(n)
    ref_lib().ref_lattice(lattice, nx, ny, nz, a0, x.ctypes.data, y.ctypes.data, z.ctypes.data)
    return x, y, z


def ref_prismatic(ref_loops, spacing, x, y, z, box, apply=None, frank=None, a0=0.0):
    """Code/main.cpp:586-687 driven over the reference's prismaticSlab."""
    lib = ref_lib()
    nl = len(ref_loops)
    handles = (c_void_p * max(1, nl))(*[rl.h for rl in ref_loops])
    sp = np.ascontiguousarray(spacing, dtype=np.float64)
    ap = np.ascontiguousarray(apply if apply is not None else [1] * nl, dtype=np.int32)
    fr = np.ascontiguousarray(frank if frank is not None else [0] * nl, dtype=np.int32)

    def fn(x_, y_, z_, n, box_, *rest):
        return lib.ref_prismatic_step(handles, sp.ctypes.data, ap.ctypes.data, fr.ctypes.data, a0,
                                      nl, x_, y_, z_, n, box_, *rest)
    return _prismatic_call(fn, x, y, z, ref_loops, box)


class RefGeometry:
    """The geometry calls of disco_b200.workloads answered by the reference's
    own code (oracle/_ref: generateLattice, snapToMidPlane, regularPolygon and
    the loop class), so that a workload can be built without this library's
    geometry: workloads.fcc_random(geom=RefGeometry) and so on.  LoopData is
    filled as Code/main.cpp:689-711 fills it."""
    BCC, FCC = 0, 1

    @staticmethod
    def lattice(kind, nx, ny, nz, a0):
        return ref_lattice(kind, nx, ny, nz, a0)

    @staticmethod
    def snap(center, n, a0, nx, ny, nz, kind):
        return ref_snap(center, n, a0, nx, ny, nz, kind)

    @staticmethod
    def regular_polygon(sides, R, m, n, vertex_dir=None):
        return ref_regular_polygon(sides, R, m, n, vertex_dir)

    @staticmethod
    def circle_eps_for_chords(radius, chords):
        lo = 1.0 - np.cos(np.pi / chords)
        hi = 1.0 - np.cos(np.pi / (chords - 1))
        return radius * 0.5 * (lo + hi)

    class Loop:
        def __init__(self, ref):
            self.ref = ref
            self._info = ref.info()

        @staticmethod
        def circle(da, radius, c, m, n, a0):
            return RefGeometry.Loop(RefLoop(0, da, c, m, n, a0, radius=radius))

        @staticmethod
        def rectangle(da, half_m, half_p, corner_r, c, m, n, a0, side=None):
            return RefGeometry.Loop(RefLoop(1, da, c, m, n, a0, half_m=half_m, half_p=half_p,
                                            corner_r=corner_r, side=side))

        @staticmethod
        def polygon(da, verts, corner_r, c, m, n, a0, axis=None):
            return RefGeometry.Loop(RefLoop(3, da, c, m, n, a0, corner_r=corner_r, side=axis,
                                            verts=np.asarray(verts, dtype=np.float64).reshape(-1, 3)))

        @property
        def center(self):
            return np.array(self._info["c"])

        def polyline(self, eps):
            return self.ref.polyline(eps)

        def _phys(self, dS):
            from disco_b200.backend import LoopPhys
            i = self._info
            return LoopPhys(*i["b"], *i["m"], *i["n"], dS)

        def line_data(self, eps=None, vertices=None):
            from disco_b200.backend import LoopData
            P = vertices if vertices is not None else self.polyline(eps)
            _, dS = self.ref.loopons()
            c = self.center
            return LoopData(phys=self._phys(dS), line=True, vx=P[:, 0].copy(), vy=P[:, 1].copy(),
                            vz=P[:, 2].copy(), cx=c[0], cy=c[1], cz=c[2])

        def loopon_data(self):
            from disco_b200.backend import LoopData
            L, dS = self.ref.loopons()
            return LoopData(x=L[:, 0].copy(), y=L[:, 1].copy(), z=L[:, 2].copy(), phys=self._phys(dS))

        def slab_loop(self, spacing, apply=True, frank=False, a0=0.0):
            return None          # the reference's matter step takes the loop object itself
