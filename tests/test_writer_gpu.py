"""The output writer on the device: the XYZ and LAMMPS atom lines of the final
positions, byte for byte equal to the oracle's (the reference's C++ stream
formatting, fixed, 8 decimals): random positions, exact ties (odd multiples of
1/512 sit half-way between two 8-decimal values), signed zeros, tiny and large
magnitudes; the short-buffer error; and the chain finalize_resident ->
format_atoms on a matter-step workload."""
import ctypes

import numpy as np
import pytest

import oracle as O
from disco_b200 import _capi as C
from disco_b200 import prismatic as P
from disco_b200 import workloads as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _format(fmt, element, pos):
    lib = C.cuda_lib()
    n = pos.shape[1]
    need = ctypes.c_int64()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = lib.disco_b200_format_atoms(fmt, element.encode(), pos[0].data_ptr(), pos[1].data_ptr(),
                                     pos[2].data_ptr(), n, None, 0, ctypes.byref(need), s)
    assert st == C.DISCO_ELIMIT and need.value > 0
    out = torch.zeros(need.value, dtype=torch.uint8, device="cuda")
    got = ctypes.c_int64()
    C.check(lib.disco_b200_format_atoms(fmt, element.encode(), pos[0].data_ptr(), pos[1].data_ptr(),
                                        pos[2].data_ptr(), n, out.data_ptr(), need.value, ctypes.byref(got), s),
            lib)
    torch.cuda.synchronize()
    assert got.value == need.value
    return bytes(out.cpu().numpy())


def _values(seed, n):
    rng = np.random.default_rng(seed)
    v = np.concatenate([rng.uniform(0.0, 542.25, n), rng.uniform(-300.0, 300.0, n // 4),
                        np.arange(1, 2 * (n // 4), 2) / 512.0, -np.arange(1, 200, 2) / 512.0,
                        np.array([0.0, -0.0, -1e-12, 1e-9, 5e-9, 2.5e-8, 1e-300, 9.9e10, -7.5e9, 1.0, 99999999.5])])
    rng.shuffle(v)
    v = v[: (len(v) // 3) * 3]
    return v.reshape(3, -1)


@pytest.mark.parametrize("n", [7, 1024, 5000, 300000])
def test_xyz_and_lammps_lines_match_the_oracle(n):
    v = _values(n, n)
    pos = torch.tensor(v, dtype=torch.float64, device="cuda")
    assert _format(0, "Fe", pos) == O.format_atoms(0, "Fe", v[0], v[1], v[2])
    a = np.abs(v)
    assert _format(1, "Fe", torch.tensor(a, dtype=torch.float64, device="cuda")) == \
        O.format_atoms(1, "Fe", a[0], a[1], a[2])


def test_nonfinite_is_rejected():
    lib = C.cuda_lib()
    pos = torch.tensor([[1.0, float("nan")], [0.0, 0.0], [0.0, 0.0]], dtype=torch.float64, device="cuda")
    b = ctypes.c_int64()
    st = lib.disco_b200_format_atoms(0, b"Fe", pos[0].data_ptr(), pos[1].data_ptr(), pos[2].data_ptr(), 2,
                                     None, 0, ctypes.byref(b), None)
    assert st == C.DISCO_EINVAL


def test_finalize_then_format_matches_the_reference_epilogue_and_writer():
    lib = C.cuda_lib()
    w = W.bcc_prismatic(cells=16, rmin=6.0, rmax=14.0, n_inter=2, n_vac=2)
    r = P.prismatic(w.x, w.y, w.z, w.slab_loops, w.box)
    sx, sy, sz = r["survivors"]
    k = len(sx)
    rng = np.random.default_rng(1)
    u = rng.normal(0.0, 0.3, size=(3, k))
    ref = O.finalize(sx, sy, sz, u[0], u[1], u[2], r["copy_atom"], r["copy_shift"], w.box)
    nc = len(r["copy_atom"])
    dpos = torch.tensor(np.stack([sx, sy, sz]), dtype=torch.float64, device="cuda")
    du = torch.tensor(u, dtype=torch.float64, device="cuda")
    cp = np.zeros((max(1, nc), 4))
    cp[:nc, 0] = r["copy_atom"].astype(np.int64).view(np.float64) if nc else 0
    cp[:nc, 1:] = r["copy_shift"]
    dcp = torch.tensor(cp, dtype=torch.float64, device="cuda")
    fin = torch.empty((6, k + nc), dtype=torch.float64, device="cuda")
    box = (ctypes.c_double * 3)(*w.box)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    C.check(lib.disco_b200_finalize_resident(dpos[0].data_ptr(), dpos[1].data_ptr(), dpos[2].data_ptr(),
                                             du[0].data_ptr(), du[1].data_ptr(), du[2].data_ptr(), k,
                                             dcp.data_ptr(), nc, box, *[fin[i].data_ptr() for i in range(6)], s),
            lib)
    torch.cuda.synchronize()
    f = fin.cpu().numpy()
    for d in range(3):
        assert np.array_equal(f[d], ref[d])
    text = _format(0, "W", fin[:3].contiguous())
    assert text == O.format_atoms(0, "W", ref[0], ref[1], ref[2])
