"""The host input synthesis (disco_b200/csrc/geometry.cpp) against the
reference's own loop class and lattice helpers (oracle/_ref): polylines,
loopon grids, mid-plane snapping, lattices, regular polygons, contour areas and
the in-plane test must be bit-identical."""
import numpy as np
import pytest

import oracle as O
from disco_b200 import geometry as G

pytestmark = pytest.mark.skipif(not O.have_ref(), reason="reference tree not compiled here")

A0 = 3.3024
C0 = (0.3, -0.2, 0.1)

SHAPES = [
    ("circle glide", dict(shape=0, radius=8.0), lambda: G.Loop.circle(0.4, 8.0, C0, (1, -1, 1), (1, 1, 0), A0),
     (1, -1, 1), (1, 1, 0)),
    ("circle prismatic", dict(shape=0, radius=8.0),
     lambda: G.Loop.circle(0.4, 8.0, C0, (-1, -1, -1), (1, 1, 1), A0), (-1, -1, -1), (1, 1, 1)),
    ("rounded rectangle", dict(shape=1, half_m=9.0, half_p=6.0, corner_r=2.5),
     lambda: G.Loop.rectangle(0.4, 9.0, 6.0, 2.5, C0, (1, 1, 1), (1, -1, 0), A0), (1, 1, 1), (1, -1, 0)),
    ("rectangle with side", dict(shape=1, half_m=5.0, half_p=7.0, corner_r=0.0, side=(1, 1, 0)),
     lambda: G.Loop.rectangle(0.4, 5.0, 7.0, 0.0, C0, (1, 1, 1), (1, -1, 0), A0, side=(1, 1, 0)),
     (1, 1, 1), (1, -1, 0)),
    ("parallelogram", dict(shape=2, half_m=7.0, half_p=5.0, dir1=(1, 1, 1), dir2=(1, 1, -1)),
     lambda: G.Loop.parallelogram(0.4, 7.0, 5.0, (1, 1, 1), (1, 1, -1), C0, (1, 1, 1), (1, -1, 0), A0),
     (1, 1, 1), (1, -1, 0)),
]


@pytest.mark.parametrize("name,kw,make,m,n", SHAPES, ids=[s[0] for s in SHAPES])
def test_shapes_bit_identical(name, kw, make, m, n):
    kw = dict(kw)
    shape = kw.pop("shape")
    r = O.RefLoop(shape, 0.4, C0, m, n, A0, **kw)
    g = make()
    for eps in (0.001, 0.01, 0.0365, 0.3, 2.0):
        assert np.array_equal(r.polyline(eps), g.polyline(eps))
    L, dS = r.loopons()
    assert np.array_equal(L, g.loopons()) and dS == g.g.dS
    info = r.info()
    assert info["area"] == g.area()
    assert np.array_equal(info["m"], g.m) and np.array_equal(info["n"], g.n)
    assert info["b"][0] == g.bmag
    rng = np.random.default_rng(3)
    for _ in range(300):
        rel = rng.uniform(-12, 12, 3)
        assert r.contains(rel) == g.contains(rel)


@pytest.mark.parametrize("sides,corner,vdir", [(6, 0.0, (1, -1, 0)), (6, 2.0, None), (5, 1.0, None),
                                               (8, 3.0, (1, 0, -1))])
def test_polygons_bit_identical(sides, corner, vdir):
    m, n = (-1, -1, -1), (1, 1, 1)
    V1 = O.ref_regular_polygon(sides, 8.0, m, n, vdir)
    V2 = G.regular_polygon(sides, 8.0, m, n, vdir)
    assert np.array_equal(V1, V2)
    r = O.RefLoop(3, 0.4, C0, m, n, A0, corner_r=corner, verts=V1, side=vdir)
    g = G.Loop.polygon(0.4, V2, corner, C0, m, n, A0, axis=vdir)
    for eps in (0.01, 0.2):
        assert np.array_equal(r.polyline(eps), g.polyline(eps))
    L, _ = r.loopons()
    assert np.array_equal(L, g.loopons())
    assert r.info()["area"] == g.area() and r.info()["r_corner"] == g.g.r_corner


@pytest.mark.parametrize("lattice", [G.BCC, G.FCC])
def test_snap_and_lattice_bit_identical(lattice):
    rng = np.random.default_rng(11)
    for nvec in [(1, 1, 0), (1, 1, 1), (1, 1, 2), (0, 0, 1), (-1, 2, 3), (2, 2, 0)]:
        for _ in range(20):
            c = rng.uniform(-30, 30, 3)
            s1 = O.ref_snap(c, nvec, 3.1, 10, 12, 14, lattice)
            s2 = G.snap(c, nvec, 3.1, 10, 12, 14, lattice)
            assert np.array_equal(s1[0], s2[0]) and s1[1] == s2[1]
    for a, b in zip(O.ref_lattice(lattice, 3, 4, 5, 3.6), G.lattice(lattice, 3, 4, 5, 3.6)):
        assert np.array_equal(a, b)


def test_circle_chord_count_rule():
    """Exactly `chords` chords for the Segment_tolerance the workloads use."""
    for R in (10.0, 17.3, 30.0, 40.0):
        eps = G.circle_eps_for_chords(R, 48)
        assert len(G.Loop.circle(1.0, R, C0, (1, -1, 0), (1, 1, 1), 3.615).polyline(eps)) == 48
    assert len(G.Loop.circle(1.0, 30.0, C0, (1, -1, 1), (1, 1, 0), 2.855).polyline(0.0365)) == 64


def test_burgers_classes_match():
    lib = O.ref_lib()
    for m, n in [((1, 1, 0), (1, -1, 1)), ((2 / 3, 2 / 3, 2 / 3), (1, 1, 1)), ((1 / 3, 1 / 3, -2 / 3), (1, 1, 1)),
                 ((1, 1, 1), (1, 1, 0)), ((0.5, 0.5, 0), (1, 1, 1))]:
        for lat in (0, 1):
            mm = np.ascontiguousarray(m, dtype=np.float64)
            nn = np.ascontiguousarray(n, dtype=np.float64)
            assert lib.ref_classify_burgers(lat, mm.ctypes.data, nn.ctypes.data) == \
                G.classify_burgers(lat, m, n)


@pytest.mark.parametrize("name", ["quadrupole", "fcc_random", "bcc_prismatic", "on_plane", "batch"])
def test_workloads_built_by_the_reference_geometry_are_identical(name):
    """The workloads built entirely by the reference's own geometry code
    (oracle.RefGeometry: generateLattice, snapToMidPlane, regularPolygon, the
    loop class) equal the ones this library builds, atom for atom and vertex
    for vertex (the reference arm of the bench uses the former)."""
    from disco_b200 import workloads as W
    make = {"quadrupole": lambda g: [W.quadrupole(cells=10, radius=8.0, geom=g)],
            "fcc_random": lambda g: [W.fcc_random(cells=12, n_circles=6, n_hex=3, n_rect=3, seed=11, geom=g)],
            "bcc_prismatic": lambda g: [W.bcc_prismatic(cells=10, rmin=4.0, rmax=8.0, geom=g)],
            "on_plane": lambda g: [W.on_plane(geom=g)],
            "batch": lambda g: W.batch(nsamples=3, edge=(5, 8), nloops=(1, 4), radius=(4.0, 8.0), geom=g)}[name]
    for a, b in zip(make(None), make(O.RefGeometry)):
        for k in "xyz":
            assert np.array_equal(getattr(a, k), getattr(b, k))
        assert len(a.loops) == len(b.loops)
        for la, lb in zip(a.loops, b.loops):
            for k in ("vx", "vy", "vz", "x", "y", "z"):
                va, vb = getattr(la, k, None), getattr(lb, k, None)
                if va is not None or vb is not None:
                    assert np.array_equal(np.asarray(va), np.asarray(vb)), k
            assert (la.cx, la.cy, la.cz) == (lb.cx, lb.cy, lb.cz)
            pa, pb = la.phys, lb.phys
            assert [pa.bx, pa.by, pa.bz, pa.mx, pa.my, pa.mz, pa.nx, pa.ny, pa.nz] == \
                [pb.bx, pb.by, pb.bz, pb.mx, pb.my, pb.mz, pb.nx, pb.ny, pb.nz]
            if not la.line:
                assert pa.dS == pb.dS
