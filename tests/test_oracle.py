"""The oracle, pinned: against the reference's own code (compiled in place into
oracle/_ref), against golden vectors the reference produced
(tests/golden/reference_vectors.npz, made by tests/golden/make_golden.py),
and against the known answers of the reference's unit tests
(Code/tests/test_barnett.cpp, Code/tests/test_prismatic.cpp)."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
from disco_b200 import _capi as C
from disco_b200 import geometry as G
from disco_b200 import workloads as W
from disco_b200.backend import LoopData, LoopPhys

GOLD = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz")
needs_ref = pytest.mark.skipif(not O.have_ref(), reason="reference tree not compiled here")


def _golden():
    return np.load(GOLD)


def _golden_loops(g, prefix):
    nv = g[prefix + "_nv"]
    phys = g[prefix + "_phys"]
    loops, o = [], 0
    for i, k in enumerate(nv):
        p = LoopPhys(*phys[i])
        if prefix + "_V" in g:
            V = g[prefix + "_V"][o:o + k]
            c = g[prefix + "_c"][i]
            loops.append(LoopData(phys=p, line=True, vx=V[:, 0].copy(), vy=V[:, 1].copy(),
                                  vz=V[:, 2].copy(), cx=c[0], cy=c[1], cz=c[2]))
        else:
            P = g[prefix + "_P"][o:o + k]
            loops.append(LoopData(x=P[:, 0].copy(), y=P[:, 1].copy(), z=P[:, 2].copy(), phys=p))
        o += k
    return loops


# ---- golden vectors (no reference needed) -----------------------------------------------

@pytest.mark.parametrize("prefix", ["line", "loopon"])
def test_oracle_matches_golden_vectors(prefix):
    g = _golden()
    xyz = g[prefix + "_xyz"]
    loops = _golden_loops(g, prefix)
    u = np.stack(O.displace(xyz[:, 0], xyz[:, 1], xyz[:, 2], loops, g[prefix + "_box"],
                            images=1, nu=0.35, nofma=True), 1)
    # contract-off restatement == contract-off reference, bit for bit
    assert np.array_equal(u, g[prefix + "_u_nofma"])
    # the reference's default flags differ only by FMA contraction
    assert np.abs(u - g[prefix + "_u"]).max() < 1e-13


def _on_plane_atoms(g, prefix):
    """Atoms exactly on some loop's plane (integer arithmetic on lattice
    coordinates: 2 (p - c) / a0 is integral for BCC sites and centres)."""
    xyz = g[prefix + "_xyz"]
    a0 = g[prefix + "_box"][0] / 12
    on = np.zeros(len(xyz), bool)
    for c, ph in zip(g[prefix + "_c"], g[prefix + "_phys"]):
        n = ph[6:9]
        q = np.rint(2 * (xyz - c) / a0)
        k = n / np.abs(n[np.abs(n) > 1e-12]).min()
        on |= np.abs(q @ np.rint(k)) == 0
    return on


def test_oracle_on_plane_matches_golden_vectors():
    """Atoms exactly on a loop's plane (inside the contour, outside it, at
    the fan apex, on fan edges): the contract-off restatement reproduces the
    contract-off reference bit for bit, so it takes the same side of the cut
    for every such atom.  The reference's two builds disagree with each other
    there, by a whole Burgers vector on some atoms: an FMA-contracted build
    rounds the solid-angle triple product differently
    (Code/barnett.hpp:69), so only the source's operation order, without
    contraction, defines the convention."""
    g = _golden()
    xyz = g["plane_xyz"]
    loops = _golden_loops(g, "plane")
    u = np.stack(O.displace(xyz[:, 0], xyz[:, 1], xyz[:, 2], loops, g["plane_box"],
                            images=1, nu=0.35, nofma=True), 1)
    assert np.array_equal(u, g["plane_u_nofma"])
    on = _on_plane_atoms(g, "plane")
    d = np.abs(g["plane_u"] - g["plane_u_nofma"]).max(1)
    assert (d > 1e-9).any() and not (d[~on] > 1e-9).any()
    bmax = max(np.linalg.norm(ph[0:3] * ph[3:6]) for ph in g["plane_phys"])
    assert d.max() <= 1.0001 * bmax


def test_oracle_prismatic_matches_golden_vectors():
    g = _golden()
    raw = g["slab_loops"].tobytes()
    nl = len(raw) // ctypes.sizeof(C.DiscoSlabLoop)
    arr = (C.DiscoSlabLoop * nl).from_buffer_copy(raw)
    xyz = g["slab_xyz"]
    r = O.prismatic(xyz[:, 0], xyz[:, 1], xyz[:, 2], list(arr), g["slab_box"])
    assert np.array_equal(r["slab_atoms"], g["slab_atoms"])
    assert np.array_equal(r["slab_side"], g["slab_side"])
    assert np.array_equal(r["new_index"], g["slab_new_index"])
    assert np.array_equal(r["copy_atom"], g["slab_copy_atom"])
    assert np.array_equal(r["copy_shift"], g["slab_copy_shift"])
    assert [len(r["survivors"][0]), len(r["slab_atoms"]), len(r["copy_atom"])] == list(g["slab_counts"])
    info = np.array([[i[0], i[1], i[2], i[3], *i[4], i[5], i[6]] for i in r["info"]])
    assert np.array_equal(info, g["slab_info"])


def test_golden_inputs_regenerate_bit_for_bit():
    """The seeded builders still produce the inputs the golden vectors were made on."""
    g = _golden()
    w = W.quadrupole(cells=10, radius=8.0, eps=0.0365)
    assert np.array_equal(np.stack([w.x, w.y, w.z], 1), g["line_xyz"])
    assert np.array_equal(np.concatenate([np.stack([l.vx, l.vy, l.vz], 1) for l in w.loops]), g["line_V"])
    w = W.bcc_prismatic(cells=10, rmin=4.0, rmax=8.0)
    assert np.array_equal(np.concatenate([np.stack([l.x, l.y, l.z], 1) for l in w.loops]), g["loopon_P"])


# ---- live reference (this container) ------------------------------------------------------

@needs_ref
@pytest.mark.parametrize("case", ["quadrupole", "fcc_random", "bcc_prismatic"])
def test_restatement_bit_identical_to_reference(case):
    """nu = 0.35, images +-1 (the reference's fixed values): the contract-off
    builds are bit-identical; the default builds differ by contraction only."""
    if case == "quadrupole":
        w = W.quadrupole(cells=8, radius=7.0, eps=0.0365)
    elif case == "fcc_random":
        w = W.fcc_random(cells=6, n_circles=3, n_hex=2, n_rect=2, seed=7)
    else:
        w = W.bcc_prismatic(cells=8, rmin=3.0, rmax=6.0, n_inter=3, n_vac=3)
    u_ref = O.ref_displace(w.x, w.y, w.z, w.loops, w.box, nofma=True)
    u_or = O.displace(w.x, w.y, w.z, w.loops, w.box, images=1, nu=0.35, nofma=True)
    for k in range(3):
        assert np.array_equal(u_ref[k], u_or[k])
    u_ref = O.ref_displace(w.x, w.y, w.z, w.loops, w.box)
    u_or = O.displace(w.x, w.y, w.z, w.loops, w.box, images=1, nu=0.35)
    floor = max(float(np.abs(u_ref[k] - u_or[k]).max()) for k in range(3))
    assert floor < 1e-13


@needs_ref
def test_pair_functions_bit_identical_to_reference():
    lib = O.ref_lib(nofma=True)
    olib = O.oracle_lib(nofma=True)
    rng = np.random.default_rng(5)
    w = W.quadrupole(cells=8, radius=7.0, eps=0.01)
    lp = w.loops[1]
    b = lp.burgers()
    for _ in range(200):
        p = rng.uniform(-12, 12, 3)
        u1, u2 = np.zeros(3), np.zeros(3)
        lib.ref_barnett_loop(*p, lp.vx.ctypes.data, lp.vy.ctypes.data, lp.vz.ctypes.data, len(lp.vx),
                             lp.cx, lp.cy, lp.cz, *b, u1.ctypes.data)
        olib.oracle_barnett_loop(*p, lp.vx.ctypes.data, lp.vy.ctypes.data, lp.vz.ctypes.data,
                                 len(lp.vx), lp.cx, lp.cy, lp.cz, *b, 0.35, u2.ctypes.data)
        assert np.array_equal(u1, u2)
        ph = LoopPhys(2.7, 2.7, 2.7, 0.57735, 0.57735, 0.57735, 0.57735, 0.57735, 0.57735, 0.2)
        d1, d2 = np.zeros(3), np.zeros(3)
        lib.ref_kroupa_pair(*p, ctypes.byref(ph.as_c()), d1.ctypes.data)
        olib.oracle_kroupa_pair(*p, ctypes.byref(ph.as_c()), 0.35, d2.ctypes.data)
        assert np.array_equal(d1, d2)


@needs_ref
def test_prismatic_restatement_matches_reference_on_config_sizes():
    """prismaticSlab + the main.cpp matter step, full 60^3 config geometry."""
    w = W.bcc_prismatic()
    refl = [O.RefLoop(0, 1.0, g.center, g.m_in, g.n_in, w.a0, radius=g.g.radius) for g in w.geom]
    r_ref = O.ref_prismatic(refl, [s.spacing for s in w.slab_loops], w.x, w.y, w.z, w.box)
    r_or = O.prismatic(w.x, w.y, w.z, w.slab_loops, w.box)
    for k in ("slab_atoms", "slab_side", "new_index", "copy_atom", "copy_shift"):
        assert np.array_equal(r_ref[k], r_or[k]), k
    # margins: no FMA contraction can move an atom across a slab or contour test
    m = O.slab_margins(w.x, w.y, w.z, w.slab_loops, w.box)
    assert m[0] > 1e-9 and m[1] > 1e-9


# ---- the reference's unit-test pins, applied to the generalised oracle ----------------------

A0 = 3.3024


def _kroupa_np(rho, m, n, bvec, dS, nu):
    """Kroupa kernel (Code/kroupa.hpp:52-73) vectorised over rows of rho."""
    k1 = 1.0 / (8.0 * np.pi * (1.0 - nu))
    r2 = np.einsum("ij,ij->i", rho, rho)
    r = np.sqrt(r2)
    br = rho @ m
    nr = rho @ n
    k2 = (1.0 - 2.0 * nu) / r
    fac = -k1 * dS / r2
    tail = 3.0 * br * nr / (r2 * r)
    bn = m @ n
    e = k2[:, None] * (np.outer(br, n) + np.outer(nr, m) - rho * bn) + tail[:, None] * rho
    return (fac[:, None] * bvec[None, :] * e).sum(0)


def _quadrature(P, c, p, m, n, bmag, nu, sub):
    """Kroupa kernel integrated over the fan triangles (c, P_k, P_k+1), each cut
    into sub^2 triangles with the 7-point degree-5 Dunavant rule
    (Code/tests/test_barnett.cpp:53-92)."""
    W7 = np.array([0.225] + [0.1323941527] * 3 + [0.1259391805] * 3)
    a1, b1, a2, b2 = 0.0597158717, 0.4701420641, 0.7974269853, 0.1012865073
    B7 = np.array([[1 / 3, 1 / 3, 1 / 3], [a1, b1, b1], [b1, a1, b1], [b1, b1, a1],
                   [a2, b2, b2], [b2, a2, b2], [b2, b2, a2]])
    pts, wts = [], []
    N = len(P)
    for t in range(N):
        e1 = (P[t] - c) / sub
        e2 = (P[(t + 1) % N] - c) / sub
        area = 0.5 * np.linalg.norm(np.cross(e1, e2))
        for i in range(sub):
            for j in range(sub - i):
                tris = [(c + i * e1 + j * e2, c + (i + 1) * e1 + j * e2, c + i * e1 + (j + 1) * e2)]
                if i + j < sub - 1:
                    tris.append((c + (i + 1) * e1 + j * e2, c + (i + 1) * e1 + (j + 1) * e2,
                                 c + i * e1 + (j + 1) * e2))
                for q0, q1, q2 in tris:
                    pts.append(B7 @ np.stack([q0, q1, q2]))
                    wts.append(W7 * area)
    X = np.concatenate(pts)
    w = np.concatenate(wts)
    bvec = bmag * np.ones(3)          # LoopPhys b = |b| per axis; m carries the direction
    k1 = 1.0 / (8.0 * np.pi * (1.0 - nu))
    rho = p[None, :] - X
    r2 = np.einsum("ij,ij->i", rho, rho)
    r = np.sqrt(r2)
    br, nr = rho @ m, rho @ n
    e = ((1.0 - 2.0 * nu) / r)[:, None] * (np.outer(br, n) + np.outer(nr, m) - rho * (m @ n)) + \
        (3.0 * br * nr / (r2 * r))[:, None] * rho
    return ((-k1 * w / r2)[:, None] * bvec[None, :] * e).sum(0)


def _test_points(c, n, m, size, count):
    """Code/tests/test_barnett.cpp:96-115: deterministic LCG, seed 2024."""
    e1 = m - (m @ n) * n
    if e1 @ e1 < 1e-12:
        e1 = np.cross(n, [1.0, 0.0, 0.0])
    if e1 @ e1 < 1e-12:
        e1 = np.cross(n, [0.0, 1.0, 0.0])
    e1 = e1 / np.linalg.norm(e1)
    e2 = np.cross(n, e1)
    seed = 2024
    pts = []

    def rnd():
        nonlocal seed
        seed = (seed * 1103515245 + 12345) & 0xFFFFFFFF
        return (seed >> 8) / float(1 << 24)
    for _ in range(count):
        a = (2 * rnd() - 1) * 1.3 * size
        b = (2 * rnd() - 1) * 1.3 * size
        h = (1 + 2 * rnd()) * (-1 if rnd() < 0.5 else 1)
        pts.append(c + a * e1 + b * e2 + h * n)
    return pts


PIN_LOOPS = [
    ("circle glide", lambda c: G.Loop.circle(0.4, 8.0, c, (1, -1, 1), (1, 1, 0), A0), 8.0, 30),
    ("circle prismatic", lambda c: G.Loop.circle(0.4, 8.0, c, (-1, -1, -1), (1, 1, 1), A0), 8.0, 30),
    ("rounded rect mixed", lambda c: G.Loop.rectangle(0.4, 9.0, 6.0, 2.5, c, (1, 1, 1), (1, -1, 0), A0), 9.0, 40),
    ("hexagon interstitial", lambda c: G.Loop.polygon(
        0.4, G.regular_polygon(6, 8.0, (-1, -1, -1), (1, 1, 1), (1, -1, 0)), 0.0, c, (-1, -1, -1),
        (1, 1, 1), A0, axis=(1, -1, 0)), 8.0, 40),
]


@pytest.mark.parametrize("nu", [0.35, 0.29])
@pytest.mark.parametrize("name,make,size,sub", PIN_LOOPS, ids=[p[0] for p in PIN_LOOPS])
def test_barnett_pins(name, make, size, sub, nu):
    """test_barnett.cpp checks 1-3 (quadrature < 1e-6 A, jump -b inside and 0
    outside < 1e-5 A, apex/start invariance < 1e-11 A) on the oracle, at the
    reference's nu and at a nu the reference cannot run."""
    c = np.array([0.3, -0.2, 0.1])
    lp = make(c)
    P = lp.polyline(0.01)
    m, n, bm = lp.m, lp.n, lp.bmag
    b = bm * m
    err = 0.0
    for p in _test_points(c, n, m, size, 4):
        ul = O.barnett_loop(p, P, c, b, nu)
        uq = _quadrature(P, c, p, m, n, bm, nu, sub)
        err = max(err, np.abs(ul - uq).max())
    assert err < 1e-6
    h = 1e-7
    jump = 0.0
    for side in (0, 1):
        q = c.copy()
        if side == 1:
            e = np.cross(n, [0.3, 0.5, 0.8])
            q = q + 3.0 * size * e / np.linalg.norm(e)
        up = O.barnett_loop(q + h * n, P, c, b, nu)
        um = O.barnett_loop(q - h * n, P, c, b, nu)
        expect = -b if side == 0 else np.zeros(3)
        jump = max(jump, np.abs(up - um - expect).max())
    assert jump < 1e-5
    k = len(P) // 3
    Pr = np.concatenate([P[k:], P[:k]])
    e = np.cross(n, [0.7, -0.2, 0.4])
    c2 = c + 0.25 * size * e / np.linalg.norm(e)
    inv = max(np.abs(O.barnett_loop(p, P, c, b, nu) - O.barnett_loop(p, Pr, c2, b, nu)).max()
              for p in _test_points(c, n, m, size, 6))
    assert inv < 1e-11


def test_loopon_sum_converges_to_line_integral():
    """test_barnett.cpp check 4: the loopon sum of a sharp prismatic hexagon
    approaches the line integral monotonically as da -> 0, below 2e-3 A."""
    m, n, c = (-1, -1, -1), (1, 1, 1), np.array([0.2, -0.1, 0.3])
    prev = 1e9
    for da in (0.8, 0.4, 0.2):
        lp = G.Loop.polygon(da, G.regular_polygon(6, 10.0, m, n), 0.0, c, m, n, A0)
        P = lp.polyline(0.01)
        L = lp.loopons()
        mh, nh, bm = lp.m, lp.n, lp.bmag
        err = 0.0
        for p0 in _test_points(c, nh, mh, 10.0, 10):
            s = (p0 - c) @ nh
            shift = (1.5 - s if s > 0 else -1.5 - s) if abs(s) < 1.5 else 0.0
            p = p0 + shift * nh
            ul = O.barnett_loop(p, P, c, bm * mh, 0.35)
            uk = _kroupa_np(p[None, :] - L, mh, nh, bm * np.ones(3), lp.g.dS, 0.35)
            err = max(err, np.abs(ul - uk).max())
        assert err < prev
        prev = err
    assert prev < 6e-3   # da = 0.2 here; the reference reaches < 2e-3 at da = 0.1


def test_far_field_is_one_loopon():
    """test_barnett.cpp check 5: a small loop seen from 105 A is one loopon of
    its area (relative difference < 1e-3)."""
    m, n, c = (1, -1, 1), (1, 1, 0), np.zeros(3)
    lp = G.Loop.circle(0.1, 2.0, c, m, n, A0)
    P = lp.polyline(0.001)
    p = np.array([60.0, -35.0, 80.0])
    ul = O.barnett_loop(p, P, c, lp.bmag * lp.m, 0.35)
    uk = O.kroupa_pair(p, LoopPhys(lp.bmag, lp.bmag, lp.bmag, *lp.m, *lp.n, lp.area()), 0.35)
    assert np.abs(ul - uk).max() / np.abs(uk).max() < 1e-3


def test_prismatic_pins_on_config_geometry():
    """test_prismatic.cpp checks on the oracle's slabs of the 60^3 config:
    k = 3 planes of BCC {111}, slab atom count within 15 % of rho A |b.n|,
    every atom inside the slab bounds with the side of its s."""
    w = W.bcc_prismatic()
    r = O.prismatic(w.x, w.y, w.z, w.slab_loops, w.box)
    rho = w.n / np.prod(w.box)
    for l, (typ, planes, height, spacing, b, off, cnt) in enumerate(r["info"]):
        g = w.geom[l]
        assert planes == 3 and abs(height - w.a0 * np.sqrt(3) / 2) < 1e-12
        assert typ == (C.MATTER_VACANCY if g.m @ g.n > 0 else C.MATTER_INTERSTITIAL)
        nomin = rho * g.area() * height
        assert abs(cnt - nomin) < 0.15 * nomin
        idx = r["slab_atoms"][off:off + cnt]
        assert np.all(np.diff(idx) > 0)
        rel = np.stack([w.x[idx], w.y[idx], w.z[idx]], 1) - g.center
        rel -= np.array(w.box) * np.floor(rel / np.array(w.box) + 0.5)
        s = rel @ g.n
        t = s / spacing
        assert np.all((t >= -1) & (t < 2))
        assert np.array_equal(r["slab_side"][off:off + cnt], np.where(s > 0, 1, -1))


def test_oracle_writer_lines_match_correctly_rounded_formatting():
    """The oracle's writer lines (the reference's C++ stream formatting) equal
    Python's correctly rounded '%.8f' on the same doubles, ties included."""
    rng = np.random.default_rng(3)
    v = np.concatenate([rng.uniform(-600, 600, 3000), np.arange(1, 4001, 2) / 512.0,
                        np.array([0.0, -0.0, -1e-12, 1e-9, 5e-9, 2.5e-8, 123456789.123456789])])
    v = v[: (len(v) // 3) * 3]
    x, y, z = v[0::3], v[1::3], v[2::3]
    got = O.format_atoms(0, "Fe", x, y, z).decode()
    want = "".join(f"Fe {a:.8f} {b:.8f} {c:.8f}\n" for a, b, c in zip(x, y, z))
    assert got == want
    got = O.format_atoms(1, "Fe", np.abs(x), np.abs(y), np.abs(z)).decode()
    want = "".join(f"{k + 1} 1 {a:.8f} {b:.8f} {c:.8f}\n"
                   for k, (a, b, c) in enumerate(zip(np.abs(x), np.abs(y), np.abs(z))))
    assert got == want
