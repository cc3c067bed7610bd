"""The kernels' own FP64 math routines against CUDA's functions (torch on the
same GPU): 1/sqrt(x) and 1/x within 1 ulp of CUDA's correctly rounded results
(the displacement kernels then stay within 1e-9 A of the oracle, which the
parity tests check end to end); the far-field series of 2 atanh(t) within
3 ulps (6.7e-16 relative) of CUDA's atanh, itself within 2 ulps, over each
tier's range.  Also the device lattice builder, bit-identical to the host
restatement of generateLattice."""
import ctypes

import numpy as np
import pytest

from disco_b200 import _capi as C

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _run(fn, x):
    lib = C.cuda_lib()
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    yd = torch.empty_like(xd)
    C.check(lib.disco_b200_math_check(fn, xd.data_ptr(), yd.data_ptr(), xd.numel(),
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), lib)
    torch.cuda.synchronize()
    return xd, yd


def _ulps(a, b):
    """|a - b| in units of b's last place."""
    a, b = a.cpu().numpy(), b.cpu().numpy()
    return np.abs(a - b) / np.spacing(np.abs(b))


def _samples(seed=0):
    rng = np.random.default_rng(seed)
    return np.concatenate([10.0 ** rng.uniform(-8, 12, 200000), rng.uniform(0.5, 2.0, 100000),
                           rng.uniform(1.0, 4.0e7, 100000), np.array([1.0, 2.0, 4.0, 0.25, 3.0])])


def test_rsqrt_within_one_ulp_of_cuda():
    x, y = _run(0, _samples())
    assert _ulps(y, torch.rsqrt(x)).max() <= 2.0           # both are within 1 ulp of 1/sqrt(x)


def test_reciprocal_within_one_ulp_of_division():
    x, y = _run(1, _samples(1))
    assert _ulps(y, 1.0 / x).max() <= 1.0


@pytest.mark.parametrize("fn,tmax", [(2, 0.11), (3, 0.054), (4, 0.012)])
def test_series_matches_atanh(fn, tmax):
    rng = np.random.default_rng(fn)
    t = np.concatenate([rng.uniform(0.0, tmax, 200000), np.array([tmax, 1e-300, 1e-12])])
    x, y = _run(fn, t)
    ref = 2.0 * torch.atanh(x)
    rel = ((y - ref).abs() / ref.abs().clamp_min(1e-300)).max().item()
    assert rel <= 3 * 2.0 ** -52


@pytest.mark.parametrize("kind,a0,cells", [(1, 3.615, (37, 38, 39)), (0, 2.855, (40, 41, 42)),
                                           (0, 3.165, (60, 60, 60))])
def test_device_lattice_is_bit_identical_to_the_host_build(kind, a0, cells):
    from disco_b200 import geometry as G
    lib = C.cuda_lib()
    x, y, z = G.lattice(kind, *cells, a0)
    d = torch.full((3, len(x)), float("nan"), dtype=torch.float64, device="cuda")
    C.check(lib.disco_b200_lattice(kind, *cells, a0, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), lib)
    got = d.cpu().numpy()
    assert np.array_equal(got[0], x) and np.array_equal(got[1], y) and np.array_equal(got[2], z)
