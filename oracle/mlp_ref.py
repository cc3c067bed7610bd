"""ORACLE — test infrastructure only.  CPU reference of the learned form's
network (14 -> 128 -> 128 -> 128 -> 3, SiLU) for checking the GPU forward
pass and gradients.  It rounds exactly what the GPU kernels round to BF16 (the
operands of every matrix product: features, weights, activations, incoming
gradients) and computes everything else in FP64, so the comparison isolates
the kernels' arithmetic from the precision choice."""
import numpy as np

KIN, KHID, KOUT, KIN_REAL, KOUT_REAL = 16, 128, 16, 14, 3
OFF = {}
_o = 0
for name, size in (("W1", KHID * KIN), ("b1", KHID), ("W2", KHID * KHID), ("b2", KHID), ("W3", KHID * KHID),
                   ("b3", KHID), ("W4", KOUT * KHID), ("b4", KOUT)):
    OFF[name] = (_o, size)
    _o += size
NPARAMS = _o


def bf16(x):
    """Round to bfloat16 (nearest, ties to even) and back to float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    out = {}
    for k, (o, s) in OFF.items():
        v = np.asarray(p[o:o + s], dtype=np.float64)
        if k == "W1":
            v = v.reshape(KHID, KIN)
        elif k in ("W2", "W3"):
            v = v.reshape(KHID, KHID)
        elif k == "W4":
            v = v.reshape(KOUT, KHID)
        out[k] = v
    return out


def silu(x):
    return x / (1.0 + np.exp(-x))


def dsilu(x):
    s = 1.0 / (1.0 + np.exp(-x))
    return s * (1.0 + x * (1.0 - s))


def forward_f64(p, X):
    """The network without any BF16 rounding (what the weights mean)."""
    P = unpack(p)
    h = np.asarray(X, dtype=np.float64)
    for W, b in (("W1", "b1"), ("W2", "b2"), ("W3", "b3")):
        h = silu(h @ P[W].T + P[b])
    return h @ P["W4"].T + P["b4"]


def forward(p, X):
    P = unpack(p)
    x0 = bf16(X)
    pre1 = x0 @ bf16(P["W1"]).T + P["b1"]
    h1 = bf16(silu(pre1))
    pre2 = h1 @ bf16(P["W2"]).T + P["b2"]
    h2 = bf16(silu(pre2))
    pre3 = h2 @ bf16(P["W3"]).T + P["b3"]
    h3 = bf16(silu(pre3))
    y = h3 @ bf16(P["W4"]).T + P["b4"]
    return y, (x0, pre1, h1, pre2, h2, pre3, h3)


def grads(p, X, T):
    """(loss, gradient vector) of the mean squared error over the 3 outputs."""
    P = unpack(p)
    n = X.shape[0]
    y, (x0, pre1, h1, pre2, h2, pre3, h3) = forward(p, X)
    d = y[:, :KOUT_REAL] - T
    loss = float((d ** 2).sum() / n)
    dy = np.zeros_like(y)
    dy[:, :KOUT_REAL] = 2.0 * d / n
    dy32 = dy.astype(np.float32).astype(np.float64)
    dyb = bf16(dy32)
    g = {}
    g["W4"] = (dyb.T @ h3) * (np.arange(KOUT)[:, None] < KOUT_REAL)
    g["b4"] = dy32.sum(0) * (np.arange(KOUT) < KOUT_REAL)
    dpre3 = (dyb @ bf16(P["W4"])) * dsilu(pre3)
    g["W3"] = bf16(dpre3).T @ h2
    g["b3"] = dpre3.sum(0)
    dpre2 = (bf16(dpre3) @ bf16(P["W3"])) * dsilu(pre2)
    g["W2"] = bf16(dpre2).T @ h1
    g["b2"] = dpre2.sum(0)
    dpre1 = (bf16(dpre2) @ bf16(P["W2"])) * dsilu(pre1)
    g["W1"] = (bf16(dpre1).T @ x0) * (np.arange(KIN)[None, :] < KIN_REAL)
    g["b1"] = dpre1.sum(0)
    out = np.zeros(NPARAMS)
    for k, (o, s) in OFF.items():
        out[o:o + s] = g[k].ravel()
    return loss, out
