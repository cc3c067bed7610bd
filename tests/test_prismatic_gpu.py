"""The GPU matter step, bit for bit: slab atoms (ascending), sides, the
new-index map, compacted survivors and the interstitial copies must equal the
oracle's (contract-off build, itself pinned to the reference); the output
epilogue must equal the oracle's too."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
from disco_b200 import _capi as C
from disco_b200 import geometry as G
from disco_b200 import prismatic as P
from disco_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz")


def _same(r, q):
    for k in ("slab_atoms", "slab_side", "new_index", "copy_atom", "copy_shift"):
        assert np.array_equal(r[k], q[k]), k
    for a, b in zip(r["survivors"], q["survivors"]):
        assert np.array_equal(a, b)
    assert r["info"] == q["info"]


def test_golden_vectors_from_the_reference():
    g = np.load(GOLD)
    raw = g["slab_loops"].tobytes()
    nl = len(raw) // ctypes.sizeof(C.DiscoSlabLoop)
    loops = list((C.DiscoSlabLoop * nl).from_buffer_copy(raw))
    xyz = g["slab_xyz"]
    r = P.prismatic(xyz[:, 0], xyz[:, 1], xyz[:, 2], loops, g["slab_box"])
    assert np.array_equal(r["slab_atoms"], g["slab_atoms"])
    assert np.array_equal(r["slab_side"], g["slab_side"])
    assert np.array_equal(r["new_index"], g["slab_new_index"])
    assert np.array_equal(r["copy_atom"], g["slab_copy_atom"])
    assert np.array_equal(r["copy_shift"], g["slab_copy_shift"])


def test_full_size_bcc_prismatic():
    """The 60^3 config (432 000 atoms, 16 loops, 3-plane slabs)."""
    w = W.bcc_prismatic()
    _same(P.prismatic(w.x, w.y, w.z, w.slab_loops, w.box),
          O.prismatic(w.x, w.y, w.z, w.slab_loops, w.box))


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_overlapping_slabs_many_loops(seed):
    """Dense overlapping vacancy and interstitial slabs: atoms removed twice,
    copies of removed atoms dropped, ragged atom counts."""
    w = W.bcc_prismatic(cells=14, rmin=5.0, rmax=14.0, n_inter=20, n_vac=20, seed=seed)
    k = w.n - 37 * seed
    x, y, z = w.x[:k], w.y[:k], w.z[:k]
    _same(P.prismatic(x, y, z, w.slab_loops, w.box), O.prismatic(x, y, z, w.slab_loops, w.box))


def test_overlapping_slabs_large_grid():
    """Dense overlapping slabs on a box large enough (128 000 atoms, more than
    64 CTAs) that the CTA counts are scanned by one CTA per category, with a
    ragged end."""
    w = W.bcc_prismatic(cells=40, rmin=5.0, rmax=14.0, n_inter=24, n_vac=24, seed=7)
    k = w.n - 77
    x, y, z = w.x[:k], w.y[:k], w.z[:k]
    _same(P.prismatic(x, y, z, w.slab_loops, w.box), O.prismatic(x, y, z, w.slab_loops, w.box))


def test_unwrapped_coordinates():
    """Atoms moved by whole box lengths, up to 2000 L from the box, as an
    unwrapped trajectory gives them: the minimum image decides membership
    (Code/prismatic.cpp:31-34), the FP32 pre-test cannot vouch for such atoms
    and hands every nearby loop to the exact test, and segments whose atoms
    scatter over many images overflow the warp's test queue.  Atom sets and
    the survivors' (unwrapped) positions bit-exact with the oracle."""
    w = W.bcc_prismatic(cells=12, rmin=4.0, rmax=10.0, n_inter=6, n_vac=6, seed=11)
    rng = np.random.default_rng(12)
    k = rng.choice([-2000, -3, -1, 0, 0, 0, 1, 2, 2000], size=(3, w.n))
    x = w.x + k[0] * w.box[0]
    y = w.y + k[1] * w.box[1]
    z = w.z + k[2] * w.box[2]
    r = P.prismatic(x, y, z, w.slab_loops, w.box)
    _same(r, O.prismatic(x, y, z, w.slab_loops, w.box))
    assert len(r["slab_atoms"]) > 0


def _shape_loops(a0, cells, lattice):
    """Every loop shape of the reference: circles, rounded rectangles,
    parallelograms, sharp and rounded polygons, on prismatic and mixed systems."""
    loops = []
    specs = [
        lambda c: G.Loop.circle(1.0, 9.0, c, (1, 1, 1), (1, 1, 1), a0),
        lambda c: G.Loop.rectangle(1.0, 9.0, 6.0, 2.5, c, (-1, -1, -1), (1, 1, 1), a0),
        lambda c: G.Loop.parallelogram(1.0, 7.0, 5.0, (1, -1, 0), (1, 0, -1), c, (1, 1, 1), (1, 1, 1), a0),
        lambda c: G.Loop.polygon(1.0, G.regular_polygon(6, 8.0, (-1, -1, -1), (1, 1, 1)), 0.0, c,
                                 (-1, -1, -1), (1, 1, 1), a0),
        lambda c: G.Loop.polygon(1.0, G.regular_polygon(5, 9.0, (1, 1, 1), (1, 1, 1)), 2.0, c,
                                 (1, 1, 1), (1, 1, 1), a0),
        lambda c: G.Loop.circle(1.0, 7.0, c, (1, 1, 1), (1, 1, 0), a0),     # mixed 1/2[111] on (110)
    ]
    rng = np.random.default_rng(8)
    L = cells * a0
    for make in specs:
        for _ in range(2):
            lp = make(np.zeros(3))
            n = lp.n_in
            cs, d = G.snap(rng.uniform(-L / 2, L / 2, 3), n, a0, cells, cells, cells, lattice)
            lp = make(cs)
            loops.append(lp.slab_loop(d, apply=True))
    return loops


def test_every_shape():
    a0, cells = 3.165, 16
    x, y, z = G.lattice(G.BCC, cells, cells, cells, a0)
    box = (cells * a0,) * 3
    loops = _shape_loops(a0, cells, G.BCC)
    _same(P.prismatic(x, y, z, loops, box), O.prismatic(x, y, z, loops, box))


def test_fcc_frank_copies_and_apply_flag():
    """FCC Frank loops (b = a0/3<111>) get the Shockley copy shift
    (Code/lattice.hpp:239-256); apply = 0 (Matter: none) selects nothing."""
    a0, cells = 3.615, 12
    x, y, z = G.lattice(G.FCC, cells, cells, cells, a0)
    box = (cells * a0,) * 3
    loops = []
    rng = np.random.default_rng(4)
    for k in range(6):
        m = (-2 / 3, -2 / 3, -2 / 3) if k % 2 == 0 else (2 / 3, 2 / 3, 2 / 3)
        cs, d = G.snap(rng.uniform(-box[0] / 2, box[0] / 2, 3), (1, 1, 1), a0, cells, cells, cells, G.FCC)
        lp = G.Loop.circle(1.0, 8.0, cs, m, (1, 1, 1), a0)
        loops.append(lp.slab_loop(d, apply=k != 3, frank=True, a0=a0))
    r = P.prismatic(x, y, z, loops, box)
    _same(r, O.prismatic(x, y, z, loops, box))
    assert r["info"][3][6] == 0 and r["info"][3][0] == C.MATTER_NONE
    if len(r["copy_shift"]):
        # the Frank shift is not a multiple of b: it has an in-plane part
        n = np.ones(3) / np.sqrt(3)
        inplane = r["copy_shift"] - np.outer(r["copy_shift"] @ n, n)
        assert np.abs(inplane).max() > 0.1


def test_glide_loops_and_empty_inputs():
    w = W.quadrupole(cells=8, radius=6.0, eps=0.0365)
    loops = [g.slab_loop(1.0) for g in w.geom]           # b.n = 0: nothing selected
    r = P.prismatic(w.x, w.y, w.z, loops, w.box)
    assert len(r["slab_atoms"]) == 0 and len(r["copy_atom"]) == 0
    assert np.array_equal(r["new_index"], np.arange(w.n, dtype=np.int32))
    assert np.array_equal(r["survivors"][0], w.x)
    r = P.prismatic(np.zeros(0), np.zeros(0), np.zeros(0), loops, w.box)
    assert len(r["new_index"]) == 0


def test_non_integer_plane_count_is_rejected():
    """|b.n| / d not an integer: the reference aborts (Code/prismatic.cpp:50-56)."""
    w = W.bcc_prismatic(cells=6, rmin=3.0, rmax=5.0, n_inter=1, n_vac=1)
    s = w.slab_loops[0]
    s.spacing = s.spacing * 1.37
    with pytest.raises(C.DiscoError) as e:
        P.prismatic(w.x, w.y, w.z, [s], w.box)
    assert e.value.status == C.DISCO_EPLANES


def test_finalize_matches_oracle():
    w = W.bcc_prismatic(cells=10, rmin=4.0, rmax=8.0)
    r = O.prismatic(w.x, w.y, w.z, w.slab_loops, w.box)
    xs, ys, zs = r["survivors"]
    rng = np.random.default_rng(2)
    u = [rng.normal(scale=0.7, size=len(xs)) for _ in range(3)]
    got = P.finalize(xs, ys, zs, *u, r["copy_atom"], r["copy_shift"], w.box)
    ref = O.finalize(xs, ys, zs, *u, r["copy_atom"], r["copy_shift"], w.box)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
