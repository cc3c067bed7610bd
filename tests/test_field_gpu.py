"""Parity of the CUDA displacement kernels with the oracle, through the C-ABI.

Tolerance: 1e-9 A per component (the plain FP64 drop-in's bar).  Small
workloads are compared atom for atom; full-size workloads on a seeded atom
subsample (the oracle finishes in seconds), plus size-independent properties
(linearity in b, the -b jump across a cut, image-split invariance)."""
import numpy as np
import pytest

import oracle as O
from disco_b200 import backend as B
from disco_b200 import workloads as W
from disco_b200.backend import AtomArrays, LoopData, LoopPhys

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _gpu(w, atoms=None, **kw):
    x, y, z = (w.x, w.y, w.z) if atoms is None else atoms
    a = AtomArrays.zeros_like_positions(x, y, z)
    B.kroupa_gpu(a, w.loops, *w.box, images=kw.pop("images", w.images), nu=kw.pop("nu", w.nu), **kw)
    return np.stack([a.ux, a.uy, a.uz], 1)


def _oracle(w, atoms=None, **kw):
    x, y, z = (w.x, w.y, w.z) if atoms is None else atoms
    return np.stack(O.displace(x, y, z, w.loops, w.box, images=kw.get("images", w.images),
                               nu=kw.get("nu", w.nu)), 1)


@pytest.mark.parametrize("images", [0, 1, 2])
def test_line_quadrupole_small(images):
    w = W.quadrupole(cells=10, radius=8.0, eps=0.0365)
    d = np.abs(_gpu(w, images=images) - _oracle(w, images=images)).max()
    assert d <= TOL


def test_line_fcc_random_small():
    w = W.fcc_random(cells=12, n_circles=6, n_hex=3, n_rect=3, seed=11)
    d = np.abs(_gpu(w) - _oracle(w)).max()
    assert d <= TOL


@pytest.mark.parametrize("images", [1, 2])
def test_loopon_prismatic_small(images):
    w = W.bcc_prismatic(cells=10, rmin=4.0, rmax=8.0)
    d = np.abs(_gpu(w, images=images) - _oracle(w, images=images)).max()
    assert d <= TOL


@pytest.mark.parametrize("split", [1, 2, 4, 8, 16, 32])
def test_image_split_does_not_change_the_sum(split):
    w = W.quadrupole(cells=8, radius=7.0, eps=0.0365)
    ref = _oracle(w)
    d = np.abs(_gpu(w, image_split=split) - ref).max()
    assert d <= TOL


def test_accumulates_into_u_and_ragged_sizes():
    """u is added to, not overwritten (Code/backend.hpp:28); atom counts that
    are not multiples of a tile."""
    w = W.quadrupole(cells=6, radius=5.0, eps=0.0365)
    ref = _oracle(w)
    for n in (1, 7, 255, 257, w.n):
        a = AtomArrays.zeros_like_positions(w.x[:n], w.y[:n], w.z[:n])
        a.ux[:] = 1.0
        a.uy[:] = -2.0
        B.kroupa_gpu(a, w.loops, *w.box, images=w.images, nu=w.nu)
        got = np.stack([a.ux - 1.0, a.uy + 2.0, a.uz], 1)
        assert np.abs(got - ref[:n]).max() <= 1e-9


def test_empty_inputs():
    w = W.quadrupole(cells=4, radius=3.0, eps=0.0365)
    a = AtomArrays.zeros_like_positions(np.zeros(0), np.zeros(0), np.zeros(0))
    B.kroupa_gpu(a, w.loops, *w.box)
    a = AtomArrays.zeros_like_positions(w.x, w.y, w.z)
    B.kroupa_gpu(a, [], *w.box)
    assert not a.ux.any() and not a.uy.any() and not a.uz.any()


def test_degenerate_segments_and_long_polylines():
    """A repeated vertex (null segment, skipped by the reference's L > 0 test)
    and a polyline longer than one table piece (> 256 segments)."""
    w = W.quadrupole(cells=8, radius=9.0, eps=0.0005)
    assert max(len(l.vx) for l in w.loops) > 256
    lp = w.loops[0]
    lp.vx = np.insert(lp.vx, 5, lp.vx[5])
    lp.vy = np.insert(lp.vy, 5, lp.vy[5])
    lp.vz = np.insert(lp.vz, 5, lp.vz[5])
    d = np.abs(_gpu(w) - _oracle(w)).max()
    assert d <= TOL


def test_mixed_line_and_loopon_loops():
    wl = W.quadrupole(cells=8, radius=6.0, eps=0.0365)
    wp = W.bcc_prismatic(cells=8, rmin=3.0, rmax=6.0, n_inter=2, n_vac=2)
    w = W.Workload("mixed", wl.x, wl.y, wl.z, wl.loops + wp.loops, wl.box, 1, 0.3, "line")
    d = np.abs(_gpu(w) - _oracle(w)).max()
    assert d <= TOL


def test_linear_in_burgers_vector():
    w = W.quadrupole(cells=8, radius=7.0, eps=0.0365)
    u1 = _gpu(w)
    for lp in w.loops:
        p = lp.phys
        lp.phys = LoopPhys(2 * p.bx, 2 * p.by, 2 * p.bz, p.mx, p.my, p.mz, p.nx, p.ny, p.nz, p.dS)
    u2 = _gpu(w)
    assert np.abs(u2 - 2 * u1).max() <= 1e-12 * max(1.0, np.abs(u1).max()) * 10


def test_jump_across_cut_is_minus_b():
    """u+ - u- = -b inside the contour, 0 outside (Code/barnett.hpp:6)."""
    w = W.quadrupole(cells=8, radius=7.0, eps=0.0365)
    lp = w.loops[0]
    c = np.array([lp.cx, lp.cy, lp.cz])
    n = np.array([lp.phys.nx, lp.phys.ny, lp.phys.nz])
    e = np.cross(n, [0.3, 0.5, 0.8])
    e /= np.linalg.norm(e)
    pts = np.array([c + 1e-7 * n, c - 1e-7 * n, c + 20 * e + 1e-7 * n, c + 20 * e - 1e-7 * n])
    one = W.Workload("one", *pts.T.copy(), [lp], w.box, 0, 0.29, "line")
    u = _gpu(one)
    b = lp.burgers()
    assert np.abs(u[0] - u[1] + b).max() < 1e-5
    assert np.abs(u[2] - u[3]).max() < 1e-5


def test_resident_plan_matches_host_call():
    torch = pytest.importorskip("torch")
    w = W.fcc_random(cells=10, n_circles=4, n_hex=2, n_rect=2, seed=3)
    host = _gpu(w)
    plan = B.Plan(w.loops, w.box, images=w.images, nu=w.nu)
    pos = torch.tensor(np.stack([w.x, w.y, w.z]), dtype=torch.float64, device="cuda")
    u = torch.zeros_like(pos)
    plan.execute(pos, u)
    plan.sync(torch.cuda.current_stream().cuda_stream)
    assert np.abs(u.cpu().numpy().T - host).max() <= 1e-12
    st = plan.stats()
    assert st["n_segments"] == sum(len(l.vx) for l in w.loops) and st["n_images"] == 125


@pytest.mark.parametrize("name", ["quadrupole", "fcc_random", "bcc_prismatic"])
def test_full_size_subsample(name):
    """The full-size workloads, all atoms on the GPU, checked on a seeded atom
    subsample against the oracle (nu and image range of each workload)."""
    w = W.FULL[name]()
    rng = np.random.default_rng(17)
    k = {"quadrupole": 400, "fcc_random": 96, "bcc_prismatic": 24}[name]
    idx = np.sort(rng.choice(w.n, size=k, replace=False))
    if name == "bcc_prismatic":
        # the loopon sum runs over the atoms that survive the matter step in
        # the full pipeline; the field itself is defined for every atom
        pass
    g = _gpu(w)
    ref = _oracle(w, atoms=(w.x[idx], w.y[idx], w.z[idx]))
    assert np.abs(g[idx] - ref).max() <= TOL


def test_largest_image_range_and_orthorhombic_box():
    """images = 8 (17^3 images, the largest the C-ABI takes) in a box with
    three different edges, line and loopon methods."""
    rng = np.random.default_rng(8)
    loops = W.fcc_random_loops(3, 8, cells=6, a0=3.615)
    box = (6 * 3.615, 5 * 3.615, 7 * 3.615)
    pos = rng.uniform(-0.5, 0.5, size=(3, 40)) * np.array(box)[:, None]
    w = W.Workload("ortho", pos[0], pos[1], pos[2], loops, box, 8, 0.31, "line")
    assert np.abs(_gpu(w) - _oracle(w)).max() <= TOL
    p = W.bcc_prismatic(cells=5, rmin=3.0, rmax=4.0, n_inter=1, n_vac=1)
    wp = W.Workload("ortho_loopons", pos[0], pos[1], pos[2], p.loops, box, 8, 0.28, "loopons")
    assert np.abs(_gpu(wp) - _oracle(wp)).max() <= TOL


def test_far_field_series_tiers_and_logarithm():
    """Atoms from 0.5 A to 2 km from one long-sided rectangle and one fine
    circle: every J0 path (logarithm, 8-, 6- and 4-term series) against the
    oracle, which always takes the logarithm."""
    from disco_b200 import geometry as G
    rect = G.Loop.rectangle(1.0, 30.0, 12.0, 0.0, (0.0, 0.0, 0.0), (1, -1, 0), (1, 1, 1), 3.615)
    circ = G.Loop.circle(1.0, 20.0, (0.0, 0.0, 0.0), (1, -1, 0), (1, 1, 1), 3.615)
    loops = [rect.line_data(vertices=rect.polyline(0.01)),
             circ.line_data(vertices=circ.polyline(G.circle_eps_for_chords(20.0, 48)))]
    r = np.concatenate([np.geomspace(0.5, 2.0e4, 300), np.geomspace(0.5, 2.0e4, 300)])
    rng = np.random.default_rng(9)
    d = rng.normal(size=(3, len(r)))
    d /= np.linalg.norm(d, axis=0)
    pos = d * r
    box = (1.0e5, 1.0e5, 1.0e5)
    w = W.Workload("tiers", pos[0], pos[1], pos[2], loops, box, 0, 0.34, "line")
    got, ref = _gpu(w), _oracle(w)
    assert np.abs(got - ref).max() <= TOL


def test_atoms_on_loop_planes_match_the_reference():
    """Atoms exactly on a loop's plane, inside and outside the contour, at the
    fan apex and on fan edges (loops centred on lattice sites, not snapped to
    mid-planes): which side of the cut such an atom takes is decided by the
    rounding of the reference's per-triangle solid angle
    (Code/barnett.hpp:69-72), and the kernel reproduces it.  Checked atom for
    atom against the reference's own output (golden vectors of its
    contract-off build, tests/golden/make_golden.py) and against the oracle at
    another nu and image range."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz"))
    w = W.on_plane()
    assert np.array_equal(np.stack([w.x, w.y, w.z], 1), g["plane_xyz"])
    got = _gpu(w, images=1, nu=0.35)
    assert np.isfinite(got).all()
    assert np.abs(got - g["plane_u_nofma"]).max() <= TOL
    ref = np.stack(O.displace(w.x, w.y, w.z, w.loops, w.box, images=2, nu=0.29, nofma=True), 1)
    assert np.abs(_gpu(w, images=2, nu=0.29) - ref).max() <= TOL
    if O.have_ref():
        live = np.stack(O.ref_displace(w.x, w.y, w.z, w.loops, w.box, nofma=True), 1)
        assert np.abs(got - live).max() <= TOL


def test_atoms_on_loop_planes_fp32c_and_batched():
    """The same on-plane atoms through the FP32 compensated form (its FP64
    near-cut pass takes the reference's side of the cut) and the batched
    form."""
    from disco_b200 import _capi as C
    from disco_b200.backend import GpuOptions
    w = W.on_plane()
    ref = np.stack(O.displace(w.x, w.y, w.z, w.loops, w.box, images=1, nu=0.35, nofma=True), 1)
    a = AtomArrays.zeros_like_positions(w.x, w.y, w.z)
    B.kroupa_gpu(a, w.loops, *w.box, GpuOptions(fp32=True), images=1, nu=0.35)
    assert np.abs(np.stack([a.ux, a.uy, a.uz], 1) - ref).max() <= 2e-5
    us, _ = B.batch_gpu([w, w], C.DISCO_FP64)
    for u in us:
        assert np.abs(np.stack(u, 1) - ref).max() <= TOL
