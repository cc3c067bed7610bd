"""The learned far-image form on the GPU.

* image_min: the exact far shells 2 <= max|n| <= images of the plan and batch
  forms against the oracle (FP64 1e-9 A, FP32C 2e-5 A), and near + far = all.
* Features: the device features against a numpy restatement of their
  definition (include/disco_b200.h, disco_far_norm).
* Fused inference: the tcgen05 far kernel against the training path's forward
  kernels on the same features (same BF16 roundings, so within 1e-3 of the
  output scale).
* What the network gains: trained here on exact far shells of random
  fcc_random-distribution loops, on held-out loops its error is a small
  fraction of the truncated sum's (dropping the far shells), it is many times
  faster than the exact far-shell sum, and faster than the far-field dipole
  (one loopon of area A per loop), which is the more accurate approximation.
* learned_displace: an untrained network fails the subsample check for every
  loop and the fallback reproduces the exact sum; a trained one passes.
"""
import numpy as np
import pytest

import oracle as O
from disco_b200 import _capi as C
from disco_b200 import backend as B
from disco_b200 import learned as Ln
from disco_b200 import workloads as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _small(cells=12, nloops=6, seed=3, n=3000):
    a0 = 3.615
    L = cells * a0
    loops = W.fcc_random_loops(nloops, seed, cells=cells, a0=a0)
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-L / 2, L / 2, size=(3, n))
    return loops, (L, L, L), pos


@pytest.mark.parametrize("precision,tol", [(C.DISCO_FP64, 1e-9), (C.DISCO_FP32C, 2e-5)])
def test_far_shells_match_oracle(precision, tol):
    loops, box, pos = _small(n=1500)
    ref = np.stack(O.displace(pos[0], pos[1], pos[2], loops, box, images=2, nu=0.34, image_min=2))
    d = torch.tensor(pos, dtype=torch.float64, device="cuda")
    u = torch.zeros_like(d)
    plan = B.Plan(loops, box, precision=precision, images=2, nu=0.34, image_min=2)
    plan.execute(d, u)
    plan.sync()
    assert np.abs(u.cpu().numpy() - ref).max() <= tol
    per = Ln.exact_far_per_loop(d, loops, box, 0.34, images=2, image_min=2, precision=precision)
    assert np.abs(per.sum(0).cpu().numpy() - ref).max() <= tol


def test_near_plus_far_is_the_whole_sum():
    loops, box, pos = _small(n=2000)
    d = torch.tensor(pos, dtype=torch.float64, device="cuda")
    parts = []
    for images, image_min in ((3, 0), (1, 0), (3, 2)):
        u = torch.zeros_like(d)
        p = B.Plan(loops, box, images=images, nu=0.34, image_min=image_min)
        p.execute(d, u)
        p.sync()
        parts.append(u)
    assert (parts[0] - parts[1] - parts[2]).abs().max().item() <= 1e-11


def _features_numpy(pos, lp, box):
    V = np.stack([lp.vx - lp.cx, lp.vy - lp.cy, lp.vz - lp.cz], 1)
    av = 0.5 * np.cross(V, np.roll(V, -1, axis=0)).sum(0)
    A = np.linalg.norm(av)
    rmax = np.linalg.norm(V, axis=1).max()
    p = lp.phys
    n = np.array([p.nx, p.ny, p.nz]) / np.linalg.norm([p.nx, p.ny, p.nz])
    b = np.array([p.bx * p.mx, p.by * p.my, p.bz * p.mz])
    bh = b / np.linalg.norm(b)
    Lref = np.cbrt(box[0] * box[1] * box[2])
    s = (pos - np.array([lp.cx, lp.cy, lp.cz])[:, None]) / np.array(box)[:, None]
    req = np.sqrt(A / np.pi)
    F = np.zeros((pos.shape[1], 16))
    F[:, 0:3] = s.T
    F[:, 3] = req / Lref
    F[:, 4:7] = n
    F[:, 7:10] = bh
    F[:, 10] = box[1] / box[0] - 1
    F[:, 11] = box[2] / box[0] - 1
    F[:, 12] = rmax / req - 1
    F[:, 13] = bh.dot(n)
    return F, np.linalg.norm(b) * A / Lref ** 2


def test_features_match_their_definition():
    loops, box, pos = _small(n=777)
    box = (box[0], box[1] * 1.1, box[2] * 0.9)
    d = torch.tensor(pos, dtype=torch.float64, device="cuda")
    X, gain = Ln.far_features(d, loops, box)
    X = X.cpu().numpy().reshape(len(loops), pos.shape[1], 16)
    for l, lp in enumerate(loops):
        F, g = _features_numpy(pos, lp, box)
        assert np.abs(X[l] - F).max() <= 2e-6, l
        assert abs(gain[l].item() - g) <= 1e-6 * g


def _norm_for(loops, box, pos):
    X, gain = Ln.far_features(pos, loops, box)
    mu, sd = X.mean(0), X.std(0)
    inv = torch.where(sd > 1e-6, 1.0 / sd.clamp_min(1e-30), torch.zeros_like(sd))
    mu[14:] = 0
    inv[14:] = 0
    return Ln.FarNorm(mu.cpu().numpy(), inv.cpu().numpy(), 0.05, 2, 2)


@pytest.mark.parametrize("n", [100, 128, 1000])
def test_fused_inference_matches_training_forward(n):
    loops, box, pos = _small(n=n)
    d = torch.tensor(pos, dtype=torch.float64, device="cuda")
    m = Ln.MLP(seed=11)
    norm = _norm_for(loops, box, d)
    per = Ln.far_apply(m, norm, d, loops, box)                       # (nloops, 3, n)
    Xs, gain = Ln.far_features(d, loops, box, norm)
    Y = m.forward(Xs)[:, :3].reshape(len(loops), n, 3).permute(0, 2, 1)
    ref = Y * gain[:, None, None] * norm.out_scale          # gain is |b| A / Lref^2 without out_scale
    m.status()
    scale = ref.abs().max().item()
    assert (per - ref).abs().max().item() <= 1e-3 * scale
    # accumulate form and loop selection
    u = torch.zeros_like(d)
    Ln.far_apply(m, norm, d, loops, box, u=u, sel=[4, 1])
    assert (u - (per[4] + per[1]).double()).abs().max().item() <= 1e-6 * scale


def test_network_gains_over_truncation_and_is_faster_than_exact():
    X, U, gain, loops, box, pos = Ln.training_set(nloops=2048, atoms=1024, seed=21)
    m, norm, hist = Ln.train(X, U, gain, 1024, epochs=6, batch=4096)
    assert hist[-1] < 0.1 * hist[0]
    held = W.fcc_random_loops(64, 99)
    rng = np.random.default_rng(7)
    L = box[0]
    ev = torch.tensor(rng.uniform(-L / 2, L / 2, size=(3, 4096)), dtype=torch.float64, device="cuda")
    r = Ln.evaluate(m, norm, ev, held, box, 0.34)
    # dropping the far shells (the method without the network) misses by r["truncation_max"]
    assert r["total_max"] < 0.25 * r["truncation_max"], r
    assert r["total_max"] < 1e-3, r
    assert r["loop_rel_rms"] < 0.2, r
    # speed: the network against the exact far-shell sum on the same pairs; each
    # figure is the best of a few calls, so that a host-side stall between the
    # two events of one call (an allocator release, say) does not count
    big = torch.tensor(rng.uniform(-L / 2, L / 2, size=(3, 32768)), dtype=torch.float64, device="cuda")
    u = torch.zeros_like(big)

    def best_ms(fn, reps):
        fn()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    p = B.Plan(held, box, images=4, nu=0.34, image_min=2)
    pd = B.Plan(Ln.dipole_loops(held), box, images=4, nu=0.34, image_min=2)

    def exact():
        p.execute(big, u)
        p.sync()

    def dipole():
        pd.execute(big, u)
        pd.sync()

    t_net = best_ms(lambda: Ln.far_apply(m, norm, big, held, box, u=u), 5)
    t_exact = best_ms(exact, 2)
    assert t_net * 20 < t_exact, (t_net, t_exact)
    # the far-field dipole (one Kroupa loopon of area A per loop, cf. the far-field
    # test of Code/tests/test_barnett.cpp) is more accurate but 702 loopon
    # evaluations per (atom, loop): the network is faster
    t_dipole = best_ms(dipole, 3)
    assert t_net * 3 < t_dipole, (t_net, t_dipole)
    assert r["dipole_max"] < r["truncation_max"], r


def test_learned_displace_falls_back_and_matches_exact():
    w = W.fcc_random(cells=40, images=4)
    loops = w.loops[:8]
    sel = np.arange(0, w.n, 37)
    d = torch.tensor(np.stack([w.x[sel], w.y[sel], w.z[sel]]), dtype=torch.float64, device="cuda")
    exact = torch.zeros_like(d)
    p = B.Plan(loops, w.box, images=4, nu=w.nu)
    p.execute(d, exact)
    p.sync()
    m = Ln.MLP(seed=2)                                   # untrained: every loop misses the check
    norm = _norm_for(loops, w.box, d)
    norm.images, norm.image_min, norm.out_scale = 4, 2, 1.0
    u = torch.zeros_like(d)
    rep = Ln.learned_displace(m, norm, d, u, loops, w.box, w.nu, check_fraction=0.05)
    assert rep["n_fallback"] == len(loops) and rep["fallback"].all()
    assert rep["n_check"] == round(0.05 * d.shape[1])
    assert (u - exact).abs().max().item() <= 2e-5
    # with tolerances no loop can miss, the network's part is what remains
    u2 = torch.zeros_like(d)
    rep2 = Ln.learned_displace(m, norm, d, u2, loops, w.box, w.nu, check_fraction=0.05, tol_loop=1e9,
                               tol_total=1e9)
    assert rep2["n_fallback"] == 0
    near = torch.zeros_like(d)
    pn = B.Plan(loops, w.box, precision=C.DISCO_FP32C, images=1, nu=w.nu)
    pn.execute(d, near)
    pn.sync()
    net = torch.zeros_like(d)
    Ln.far_apply(m, norm, d, loops, w.box, u=net)
    assert (u2 - near - net).abs().max().item() <= 1e-9 + 1e-6 * net.abs().max().item()
