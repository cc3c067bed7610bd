"""Python wrappers of the host input-synthesis library (include/disco_geometry.h):
lattices, mid-plane snapping, loop shapes, polylines and loopon grids, restated
from the reference's Code/lattice.hpp and Code/loop.cpp."""
import ctypes

import numpy as np

from . import _capi as C
from .backend import LoopData, LoopPhys

BCC, FCC = C.LATTICE_BCC, C.LATTICE_FCC


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _d3(v):
    return (ctypes.c_double * 3)(*[float(t) for t in v])


def lattice(kind, nx, ny, nz, a0):
    """generateLattice (Code/lattice.hpp:35-51): x, y, z arrays."""
    lib = C.geom_lib()
    nb = 4 if kind == FCC else 2
    n = nb * nx * ny * nz
    x, y, z = np.empty(n), np.empty(n), np.empty(n)
    got = lib.disco_geom_lattice(kind, nx, ny, nz, a0, x.ctypes.data, y.ctypes.data, z.ctypes.data)
    assert got == n
    return x, y, z


def snap(center, n, a0, nx, ny, nz, kind):
    """snapToMidPlane (Code/loop.cpp:342-374): (snapped centre, plane spacing)."""
    lib = C.geom_lib()
    out = (ctypes.c_double * 3)()
    d = ctypes.c_double()
    C.check(lib.disco_geom_snap(_d3(center), _d3(n), a0, nx, ny, nz, kind, out, ctypes.byref(d)), lib)
    return np.array(out[:]), d.value


class Loop:
    """One loop's geometry (the reference's loop class state, compress = 1).
    m_in, n_in keep the constructor's m and n as given (Miller vectors)."""

    def __init__(self, g, m_in=None, n_in=None):
        self.g = g
        self.m_in = None if m_in is None else tuple(float(t) for t in m_in)
        self.n_in = None if n_in is None else tuple(float(t) for t in n_in)

    # ---- constructors (Code/loop.cpp:58-244) ----
    @staticmethod
    def circle(da, radius, c, m, n, a0):
        g = C.DiscoGeomLoop()
        lib = C.geom_lib()
        C.check(lib.disco_geom_circle(da, radius, _d3(c), _d3(m), _d3(n), a0, ctypes.byref(g)), lib)
        return Loop(g, m, n)

    @staticmethod
    def rectangle(da, half_m, half_p, corner_r, c, m, n, a0, side=None):
        g = C.DiscoGeomLoop()
        lib = C.geom_lib()
        C.check(lib.disco_geom_rectangle(da, half_m, half_p, corner_r, _d3(c), _d3(m), _d3(n), a0,
                                         _d3(side) if side is not None else None, ctypes.byref(g)), lib)
        return Loop(g, m, n)

    @staticmethod
    def parallelogram(da, half1, half2, dir1, dir2, c, m, n, a0):
        g = C.DiscoGeomLoop()
        lib = C.geom_lib()
        C.check(lib.disco_geom_parallelogram(da, half1, half2, _d3(dir1), _d3(dir2), _d3(c), _d3(m),
                                             _d3(n), a0, ctypes.byref(g)), lib)
        return Loop(g, m, n)

    @staticmethod
    def polygon(da, verts, corner_r, c, m, n, a0, axis=None):
        g = C.DiscoGeomLoop()
        lib = C.geom_lib()
        v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
        C.check(lib.disco_geom_polygon(da, _dp(v), v.shape[0], corner_r, _d3(c), _d3(m), _d3(n), a0,
                                       _d3(axis) if axis is not None else None, ctypes.byref(g)), lib)
        return Loop(g, m, n)

    # ---- derived quantities ----
    def polyline(self, eps):
        """loop::polyline (Code/loop.cpp:536-580): (nv, 3) vertices, CCW about n."""
        lib = C.geom_lib()
        nv = lib.disco_geom_polyline(ctypes.byref(self.g), eps, None, 0)
        out = np.empty((nv, 3))
        lib.disco_geom_polyline(ctypes.byref(self.g), eps, _dp(out), nv)
        return out

    def loopons(self):
        """generateLoopons (Code/loop.cpp:253-273): (n, 3) loopon positions."""
        lib = C.geom_lib()
        n = lib.disco_geom_loopons(ctypes.byref(self.g), None, 0)
        out = np.empty((n, 3))
        lib.disco_geom_loopons(ctypes.byref(self.g), _dp(out), n)
        return out

    def area(self):
        return C.geom_lib().disco_geom_area(ctypes.byref(self.g))

    def contains(self, rel):
        return bool(C.geom_lib().disco_geom_contains(ctypes.byref(self.g), _d3(rel)))

    @property
    def center(self):
        return np.array(self.g.c[:])

    @property
    def m(self):
        return np.array(self.g.m[:])

    @property
    def n(self):
        return np.array(self.g.n[:])

    @property
    def bmag(self):
        return self.g.bmag

    def phys(self):
        """LoopPhys as Code/main.cpp:700 fills it: b = |b| per axis, unit m, n, dS."""
        g = self.g
        return LoopPhys(g.bmag, g.bmag, g.bmag, *g.m[:], *g.n[:], g.dS)

    def line_data(self, eps=None, vertices=None):
        """LoopData of the line method (Code/main.cpp:703-710)."""
        P = vertices if vertices is not None else self.polyline(eps)
        c = self.center
        return LoopData(phys=self.phys(), line=True, vx=P[:, 0].copy(), vy=P[:, 1].copy(),
                        vz=P[:, 2].copy(), cx=c[0], cy=c[1], cz=c[2])

    def loopon_data(self):
        """LoopData of the loopon method (Code/main.cpp:693-701)."""
        L = self.loopons()
        return LoopData(x=L[:, 0].copy(), y=L[:, 1].copy(), z=L[:, 2].copy(), phys=self.phys())

    def slab_loop(self, spacing, apply=True, frank=False, a0=0.0):
        """disco_slab_loop of this loop for the matter step."""
        s = C.DiscoSlabLoop()
        lib = C.geom_lib()
        C.check(lib.disco_geom_slab_loop(ctypes.byref(self.g), spacing, int(apply), int(frank), a0,
                                         ctypes.byref(s)), lib)
        return s


def regular_polygon(sides, R, m, n, vertex_dir=None):
    """regularPolygon (Code/loop.cpp:585-608): (sides, 3) in-plane offsets."""
    lib = C.geom_lib()
    out = np.empty((sides, 3))
    C.check(lib.disco_geom_regular_polygon(sides, R, _d3(vertex_dir) if vertex_dir is not None else None,
                                           _d3(m), _d3(n), _dp(out)), lib)
    return out


def classify_burgers(kind, m, n):
    return C.geom_lib().disco_geom_classify_burgers(kind, _d3(m), _d3(n))


def circle_eps_for_chords(radius, chords):
    """A Segment_tolerance for which loop::polyline cuts a circle of this radius
    into exactly `chords` chords (Code/loop.cpp:487-493,540-548)."""
    lo = 1.0 - np.cos(np.pi / chords)
    hi = 1.0 - np.cos(np.pi / (chords - 1))
    return radius * 0.5 * (lo + hi)
