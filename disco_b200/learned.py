"""Learned far-image surrogate: the network, its training and its use in the
displacement sum.

A loop's field summed over the far periodic-image shells image_min <= max|n| <=
images (702 of the 729 images of +-4 for image_min 2) is slowly converging and
smooth in the atom's position; a small network stands in for it.  MLP wraps the
C-ABI network (14 -> 128 -> 128 -> 128 -> 3, SiLU, BF16 tensor cores, FP32
accumulation and master weights, Adam), trained and evaluated by this library's
own tcgen05 kernels.  FarNorm is the feature standardisation and output scale
that go with a trained network.  training_set() draws random loops of the
fcc_random distribution and atoms uniform in its box and sums their far shells
exactly (FP64 batched form); train() fits the network on the GPU;
learned_displace() is the learned form of the displacement: exact near images,
the network's far shells, the exact far-shell sum re-checked on a random atom
subsample every call with per-loop fallback.  Tensors are torch CUDA tensors
(device memory and streams only)."""
import ctypes
import math
import os
import time
from dataclasses import dataclass, field

import numpy as np

from . import _capi as C
from . import backend as B


class MLP:
    IN, OUT, IN_REAL, OUT_REAL = 16, 16, 14, 3

    def __init__(self, seed=0):
        self._lib = C.cuda_lib()
        h = ctypes.c_void_p()
        C.check(self._lib.disco_b200_mlp_create(ctypes.c_uint64(seed), ctypes.byref(h)), self._lib)
        self._h = h
        self.nparams = self._lib.disco_b200_mlp_param_count()

    def params(self):
        out = np.empty(self.nparams, dtype=np.float32)
        C.check(self._lib.disco_b200_mlp_get_params(self._h, out.ctypes.data), self._lib)
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparams
        C.check(self._lib.disco_b200_mlp_set_params(self._h, p.ctypes.data), self._lib)

    def grads(self):
        out = np.empty(self.nparams, dtype=np.float32)
        C.check(self._lib.disco_b200_mlp_get_grads(self._h, out.ctypes.data), self._lib)
        return out

    @staticmethod
    def _stream(stream):
        import torch
        return (stream or torch.cuda.current_stream()).cuda_stream

    def forward(self, X, stream=None):
        """X: (n, 16) float32 CUDA tensor -> (n, 16) float32 (first 3 used)."""
        import torch
        assert X.dtype == torch.float32 and X.is_cuda and X.is_contiguous() and X.shape[1] == self.IN
        Y = torch.empty((X.shape[0], self.OUT), dtype=torch.float32, device=X.device)
        C.check(self._lib.disco_b200_mlp_forward(self._h, X.data_ptr(), X.shape[0], Y.data_ptr(),
                                                 ctypes.c_void_p(self._stream(stream))), self._lib)
        return Y

    def grad(self, X, T, stream=None, want_loss=True):
        """Accumulates the MSE gradient over the rows of X (n, 16) against
        T (n, 3); returns the loss (None without want_loss: no host sync)."""
        loss = ctypes.c_float()
        C.check(self._lib.disco_b200_mlp_grad(self._h, X.data_ptr(), T.data_ptr(), X.shape[0],
                                              ctypes.byref(loss) if want_loss else None,
                                              ctypes.c_void_p(self._stream(stream))),
                self._lib)
        return loss.value if want_loss else None

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0, stream=None):
        C.check(self._lib.disco_b200_mlp_adam(self._h, lr, beta1, beta2, eps, weight_decay,
                                              ctypes.c_void_p(self._stream(stream))), self._lib)

    def status(self):
        C.check(self._lib.disco_b200_mlp_status(self._h), self._lib)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.disco_b200_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- far shells ------------------------------------------------------------------------

@dataclass
class FarNorm:
    """disco_far_norm: feature k enters as (raw_k - mu[k]) * inv_sd[k]; output
    times out_scale * |b| A / Lref^2 is the far-shell displacement (A)."""
    mu: np.ndarray = field(default_factory=lambda: np.zeros(16, np.float32))
    inv_sd: np.ndarray = field(default_factory=lambda: np.ones(16, np.float32))
    out_scale: float = 1.0
    images: int = 4
    image_min: int = 2

    def as_c(self):
        c = C.DiscoFarNorm()
        for k in range(16):
            c.mu[k] = float(self.mu[k])
            c.inv_sd[k] = float(self.inv_sd[k])
        c.out_scale = float(self.out_scale)
        c.images = int(self.images)
        c.image_min = int(self.image_min)
        return c


def save(path, mlp, norm, meta=None):
    np.savez(path, params=mlp.params(), mu=norm.mu, inv_sd=norm.inv_sd, out_scale=norm.out_scale,
             images=norm.images, image_min=norm.image_min, meta=str(meta or {}))


def load(path, seed=0):
    d = np.load(path)
    m = MLP(seed=seed)
    m.set_params(d["params"])
    norm = FarNorm(d["mu"].astype(np.float32), d["inv_sd"].astype(np.float32), float(d["out_scale"]),
                   int(d["images"]), int(d["image_min"]))
    return m, norm


def _atoms(pos, u=None):
    """DiscoAtoms of device tensors pos (3, n) float64 [and u (3, n)]."""
    a = C.DiscoAtoms()
    a.x, a.y, a.z = pos[0].data_ptr(), pos[1].data_ptr(), pos[2].data_ptr()
    if u is not None:
        a.ux, a.uy, a.uz = u[0].data_ptr(), u[1].data_ptr(), u[2].data_ptr()
    a.n = pos.shape[1]
    return a


def _stream_ptr(stream=None):
    import torch
    return ctypes.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)


def far_features(pos, loops, box, norm=None, stream=None):
    """(X (nloops n, 16) float32, gain (nloops,) float32): the features of every
    (loop, atom) pair, loop-major, raw without norm."""
    import torch
    lib = C.cuda_lib()
    n = pos.shape[1]
    X = torch.empty((len(loops) * n, 16), dtype=torch.float32, device=pos.device)
    gain = torch.empty(max(1, len(loops)), dtype=torch.float32, device=pos.device)
    arr, keep = B.loop_array(loops)
    b = (ctypes.c_double * 3)(*[float(v) for v in box])
    nc = norm.as_c() if norm is not None else None
    C.check(lib.disco_b200_far_features(ctypes.byref(_atoms(pos)), arr, len(loops), b,
                                        ctypes.byref(nc) if nc is not None else None, X.data_ptr(),
                                        gain.data_ptr(), _stream_ptr(stream)), lib)
    del keep
    return X, gain[:len(loops)]


def far_apply(mlp, norm, pos, loops, box, u=None, sel=None, stream=None):
    """The network's far shells: added into u (3, n) float64, or, with u None,
    returned per loop as (nsel, 3, n) float32."""
    import torch
    lib = C.cuda_lib()
    n = pos.shape[1]
    arr, keep = B.loop_array(loops)
    b = (ctypes.c_double * 3)(*[float(v) for v in box])
    nsel = len(loops) if sel is None else len(sel)
    sel_arr = None if sel is None else (ctypes.c_int32 * max(1, nsel))(*[int(v) for v in sel])
    out = None if u is not None else torch.zeros((nsel, 3, n), dtype=torch.float32, device=pos.device)
    nc = norm.as_c()
    C.check(lib.disco_b200_far_apply(mlp._h, ctypes.byref(nc), ctypes.byref(_atoms(pos, u)), arr, len(loops), b,
                                     sel_arr, nsel, out.data_ptr() if out is not None else None,
                                     _stream_ptr(stream)), lib)
    del keep
    return out


def learned_displace(mlp, norm, pos, u, loops, box, nu, precision=C.DISCO_FP32C, check_precision=C.DISCO_FP32C,
                     check_fraction=0.01, tol_loop=1e-3, tol_total=1e-3, seed=0, stream=None):
    """The learned form: u (3, n) += exact near images + the network's far shells
    (exact for the loops that miss the check).  The check's exact far shells
    are FP32 compensated by default: within about 1e-5 A of FP64 on a whole
    sum, two orders below the tolerances, at twice the FP64 rate (pass
    check_precision=C.DISCO_FP64 for the plain FP64 sum).  Returns the report
    as a dict."""
    lib = C.cuda_lib()
    arr, keep = B.loop_array(loops)
    b = (ctypes.c_double * 3)(*[float(v) for v in box])
    o = C.DiscoLearnedOptions(precision, check_precision, nu, check_fraction, tol_loop, tol_total, seed)
    nl = len(loops)
    lerr = np.zeros(max(1, nl))
    fb = np.zeros(max(1, nl), dtype=np.int32)
    r = C.DiscoLearnedReport()
    r.loop_err = lerr.ctypes.data
    r.fallback = fb.ctypes.data
    nc = norm.as_c()
    C.check(lib.disco_b200_learned_displace(mlp._h, ctypes.byref(nc), ctypes.byref(_atoms(pos, u)), arr, nl, b,
                                            ctypes.byref(o), ctypes.byref(r), _stream_ptr(stream)), lib)
    del keep
    return {"n_check": r.n_check, "n_fallback": r.n_fallback, "launches": r.launches, "check_max": r.check_max,
            "check_rms": r.check_rms, "worst_loop": r.worst_loop, "t_check": r.t_check, "t_near": r.t_near,
            "t_far": r.t_far, "t_fallback": r.t_fallback, "loop_err": lerr[:nl].copy(),
            "fallback": fb[:nl].astype(bool)}


def exact_far_per_loop(pos, loops, box, nu, images=4, image_min=2, precision=C.DISCO_FP64):
    """(nloops, 3, n) float64: every loop's exact far-shell field at the atoms
    (batched form, one sample per loop, all on the device)."""
    import torch
    lib = C.cuda_lib()
    n = pos.shape[1]
    out = torch.zeros((len(loops), 3, n), dtype=torch.float64, device=pos.device)
    arr = (C.DiscoSample * max(1, len(loops)))()
    keep = []
    for l, lp in enumerate(loops):
        la, lk = B.loop_array([lp])
        keep += [la, lk]
        d = arr[l]
        d.atoms = C.DiscoAtoms(pos[0].data_ptr(), pos[1].data_ptr(), pos[2].data_ptr(), out[l, 0].data_ptr(),
                               out[l, 1].data_ptr(), out[l, 2].data_ptr(), n)
        d.loops = ctypes.cast(la, ctypes.c_void_p)
        d.nloops = 1
        d.images = images
        d.image_min = image_min
        d.box = C.D3(*[float(v) for v in box])
    o = B.options(precision, images, nu)
    h = ctypes.c_void_p()
    C.check(lib.disco_b200_batch_plan_create(arr, len(loops), ctypes.byref(o), ctypes.byref(h)), lib)
    try:
        s = _stream_ptr()
        C.check(lib.disco_b200_batch_plan_execute(h, s), lib)
        C.check(lib.disco_b200_batch_plan_sync(h, s), lib)
    finally:
        lib.disco_b200_batch_plan_destroy(h)
    del keep
    return out


def dipole_loops(loops):
    """Each line loop as its far-field dipole: one Kroupa loopon of the loop's
    area at its centre, same b, m and n."""
    out = []
    for lp in loops:
        V = np.stack([lp.vx - lp.cx, lp.vy - lp.cy, lp.vz - lp.cz], 1)
        A = 0.5 * np.linalg.norm(np.cross(V, np.roll(V, -1, axis=0)).sum(0))
        p = lp.phys
        phys = B.LoopPhys(p.bx, p.by, p.bz, p.mx, p.my, p.mz, p.nx, p.ny, p.nz, A)
        out.append(B.LoopData(np.array([lp.cx]), np.array([lp.cy]), np.array([lp.cz]), phys, False))
    return out


def training_set(nloops=4096, atoms=1024, seed=5, nu=0.34, cells=150, a0=3.615, images=4, image_min=2):
    """Exact far-shell samples: `nloops` random loops of the fcc_random
    distribution, each evaluated at the same `atoms` positions drawn uniformly
    in its box (so atom - centre spans the box's full range).  Returns raw
    features X (nloops atoms, 16), displacements U (nloops atoms, 3) in A,
    gains (nloops,), the loops and the box."""
    import torch
    from . import workloads as W
    loops = W.fcc_random_loops(nloops, seed, cells=cells, a0=a0)
    L = cells * a0
    box = (L, L, L)
    rng = np.random.default_rng(seed + 1000)
    pos = torch.tensor(rng.uniform(-L / 2, L / 2, size=(3, atoms)), dtype=torch.float64, device="cuda")
    U = exact_far_per_loop(pos, loops, box, nu, images, image_min)              # (nloops, 3, atoms)
    X, gain = far_features(pos, loops, box)
    U = U.permute(0, 2, 1).reshape(-1, 3).contiguous()
    return X, U, gain, loops, box, pos


def fit_norm(X, U, gain, atoms, images=4, image_min=2):
    """Feature standardisation and output scale of a training set."""
    import torch
    mu = X.mean(0)
    sd = X.std(0)
    inv = torch.where(sd > 1e-6, 1.0 / sd.clamp_min(1e-30), torch.zeros_like(sd))
    mu[14:] = 0.0
    inv[14:] = 0.0
    g = gain.repeat_interleave(atoms)[:, None]
    T = U / g
    out_scale = float(T.pow(2).mean().sqrt())
    return FarNorm(mu.float().cpu().numpy(), inv.float().cpu().numpy(), out_scale, images, image_min)


def train(X, U, gain, atoms, norm=None, epochs=8, batch=4096, lr=1e-2, lr_min=1e-5, seed=0, log=None):
    """Fits a fresh network to (X, U) with Adam on this library's tcgen05
    kernels; cosine learning-rate decay.  Returns (mlp, norm, history)."""
    import torch
    norm = norm or fit_norm(X, U, gain, atoms)
    mu = torch.tensor(norm.mu, device=X.device)
    inv = torch.tensor(norm.inv_sd, device=X.device)
    Xs = ((X - mu) * inv).float().contiguous()
    T = (U / gain.repeat_interleave(atoms)[:, None] / norm.out_scale).float().contiguous()
    m = MLP(seed=seed)
    N = Xs.shape[0]
    steps = N // batch
    total = epochs * steps
    gen = torch.Generator(device=X.device)
    gen.manual_seed(seed)
    hist = []
    t0 = time.time()
    k = 0
    for ep in range(epochs):
        perm = torch.randperm(N, device=X.device, generator=gen)
        Xp, Tp = Xs[perm], T[perm]
        acc, cnt = 0.0, 0
        for i in range(steps):
            rate = lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * k / max(1, total)))
            want = (i % 64 == 0) or i == steps - 1
            loss = m.grad(Xp[i * batch:(i + 1) * batch], Tp[i * batch:(i + 1) * batch], want_loss=want)
            m.adam(lr=rate)
            if want:
                acc += loss
                cnt += 1
            k += 1
        m.status()
        hist.append(acc / max(1, cnt))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.3e} lr {rate:.2e} ({time.time() - t0:.1f} s)")
    return m, norm, hist


def evaluate(mlp, norm, pos, loops, box, nu):
    """Per-loop far shells: network vs exact (FP64) on device atoms pos.
    Returns a dict of errors in A plus the exact and dipole fields' sizes."""
    import torch
    exact = exact_far_per_loop(pos, loops, box, nu, norm.images, norm.image_min)
    net = far_apply(mlp, norm, pos, loops, box).double()
    dip = exact_far_per_loop(pos, dipole_loops(loops), box, nu, norm.images, norm.image_min)
    d = net - exact
    tot_exact, tot_d, tot_dip = exact.sum(0), d.sum(0), (dip - exact).sum(0)
    return {
        "loop_max": float(d.abs().max()), "loop_rms": float(d.pow(2).mean().sqrt()),
        "loop_rel_rms": float(d.pow(2).mean().sqrt() / exact.pow(2).mean().sqrt()),
        "total_max": float(tot_d.abs().max()), "total_rms": float(tot_d.pow(2).mean().sqrt()),
        "truncation_max": float(tot_exact.abs().max()), "truncation_rms": float(tot_exact.pow(2).mean().sqrt()),
        "dipole_max": float(tot_dip.abs().max()), "dipole_rms": float(tot_dip.pow(2).mean().sqrt()),
    }


def cached_or_train(path, log=None, **kw):
    """Loads the network at `path` or trains one (training_set + train) and
    saves it there."""
    if path and os.path.exists(path):
        return load(path) + ({"cached": True},)
    t0 = time.time()
    X, U, gain, loops, box, pos = training_set(**{k: v for k, v in kw.items()
                                                  if k in ("nloops", "atoms", "seed", "nu", "cells", "a0")})
    t1 = time.time()
    m, norm, hist = train(X, U, gain, pos.shape[1], log=log,
                          **{k: v for k, v in kw.items() if k in ("epochs", "batch", "lr", "lr_min")})
    t2 = time.time()
    info = {"cached": False, "samples": int(X.shape[0]), "data_seconds": t1 - t0, "train_seconds": t2 - t1,
            "loss": hist}
    if path:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        save(path, m, norm, info)
    return m, norm, info


def _main():
    """python -m disco_b200.learned far --atoms N --loops L [--reps R]: the fused
    far kernel on a seeded case (random-init network, fcc_random-distribution
    loops, atoms uniform in the 150^3 FCC box), timed with CUDA events; the
    case the far kernel's ncu summaries are taken on.
    python -m disco_b200.learned train [--batch B] [--reps R]: training steps
    (forward, backward, Adam) on seeded random data, timed the same way."""
    import argparse
    import torch
    from . import workloads as W
    p = argparse.ArgumentParser()
    p.add_argument("what", choices=["far", "train"])
    p.add_argument("--atoms", type=int, default=131072)
    p.add_argument("--loops", type=int, default=64)
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--batch", type=int, default=4096)
    a = p.parse_args()
    if a.what == "train":
        # training steps on seeded random data: per-step time of grad + Adam
        torch.manual_seed(0)
        X = torch.zeros((a.batch * 8, 16), dtype=torch.float32, device="cuda")
        X[:, :14].uniform_(-1, 1)
        T = torch.stack([torch.sin(2 * X[:, 0]) * X[:, 3], X[:, 1] * X[:, 2], torch.cos(X[:, 4] + X[:, 5])], 1)
        m = MLP(seed=1)
        for i in range(8):
            m.grad(X[i * a.batch:(i + 1) * a.batch], T[i * a.batch:(i + 1) * a.batch], want_loss=False)
            m.adam(lr=1e-3)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.time()
        e0.record()
        for k in range(a.reps):
            i = k % 8
            m.grad(X[i * a.batch:(i + 1) * a.batch], T[i * a.batch:(i + 1) * a.batch], want_loss=False)
            m.adam(lr=1e-3)
        e1.record()
        torch.cuda.synchronize()
        wall = time.time() - t0
        m.status()
        print(f"training step (batch {a.batch}): {e0.elapsed_time(e1) / a.reps:.3f} ms device, "
              f"{1e3 * wall / a.reps:.3f} ms wall per step")
        return
    L = 150 * 3.615
    box = (L, L, L)
    loops = W.fcc_random_loops(a.loops, 2)
    rng = np.random.default_rng(0)
    pos = torch.tensor(rng.uniform(-L / 2, L / 2, size=(3, a.atoms)), dtype=torch.float64, device="cuda")
    u = torch.zeros_like(pos)
    m = MLP(seed=1)
    X, gain = far_features(pos[:, :4096].contiguous(), loops, box)
    mu, sd = X.mean(0), X.std(0)
    inv = torch.where(sd > 1e-6, 1.0 / sd.clamp_min(1e-30), torch.zeros_like(sd))
    mu[14:] = 0.0
    inv[14:] = 0.0
    norm = FarNorm(mu.cpu().numpy(), inv.cpu().numpy(), 0.01)
    far_apply(m, norm, pos, loops, box, u=u)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        far_apply(m, norm, pos, loops, box, u=u)
    e1.record()
    torch.cuda.synchronize()
    m.status()
    t = e0.elapsed_time(e1) * 1e-3 / a.reps
    pairs = a.atoms * a.loops
    flop = 2 * (16 * 128 + 2 * 128 * 128 + 128 * 16) * pairs
    print(f"far kernel: {a.atoms} atoms x {a.loops} loops = {pairs} pairs, {t * 1e3:.3f} ms per call, "
          f"{pairs / t:.3e} pairs/s, {flop / t / 1e12:.1f} TFLOP/s (BF16 MMA, padded shapes)")


if __name__ == "__main__":
    _main()
