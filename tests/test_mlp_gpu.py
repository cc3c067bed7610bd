"""The learned form's network on the tensor cores (tcgen05) against the CPU
oracle (oracle/mlp_ref.py): forward outputs and every parameter's gradient,
with the oracle rounding the same operands to BF16.  Tolerances: forward
2e-3 relative to the output scale, gradients 2e-2 relative per parameter block
(BF16 rounding of activations can fall on the other side of a tie when the
FP32 accumulation order differs)."""
import numpy as np
import pytest

import oracle.mlp_ref as R
from disco_b200.learned import MLP

pytestmark = pytest.mark.gpu


def _data(n, seed=0):
    rng = np.random.default_rng(seed)
    X = np.zeros((n, 16), dtype=np.float32)
    X[:, :14] = rng.uniform(-1, 1, size=(n, 14))
    T = np.stack([np.sin(2 * X[:, 0]) * X[:, 3], X[:, 1] * X[:, 2], np.cos(X[:, 4] + X[:, 5])], 1)
    return X, T.astype(np.float32)


@pytest.mark.parametrize("n", [128, 300, 4096])
def test_forward_matches_oracle(n):
    torch = pytest.importorskip("torch")
    m = MLP(seed=3)
    X, _ = _data(n)
    Y = m.forward(torch.from_numpy(X).cuda()).cpu().numpy()
    m.status()
    ref, _ = R.forward(m.params(), X)
    scale = np.abs(ref[:, :3]).max()
    assert np.abs(Y[:, :3] - ref[:, :3]).max() <= 2e-3 * scale
    assert np.abs(Y[:, 3:]).max() == 0.0          # padding outputs stay zero


@pytest.mark.parametrize("n", [256, 1000])
def test_gradients_match_oracle(n):
    torch = pytest.importorskip("torch")
    m = MLP(seed=5)
    X, T = _data(n, seed=1)
    loss = m.grad(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda())
    m.status()
    g = m.grads()
    ref_loss, ref = R.grads(m.params(), X, T)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss
    for name, (o, s) in R.OFF.items():
        a, b = g[o:o + s].astype(np.float64), ref[o:o + s]
        nb = np.linalg.norm(b)
        if nb == 0:
            assert np.abs(a).max() == 0.0, name
            continue
        assert np.linalg.norm(a - b) <= 2e-2 * nb, (name, np.linalg.norm(a - b) / nb)


def test_training_reduces_loss():
    torch = pytest.importorskip("torch")
    m = MLP(seed=7)
    X, T = _data(8192, seed=2)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    first = None
    for step in range(300):
        i = (step * 1024) % 8192
        loss = m.grad(Xd[i:i + 1024], Td[i:i + 1024])
        m.adam(lr=2e-3)
        first = loss if first is None else first
    m.status()
    assert loss < 0.1 * first
