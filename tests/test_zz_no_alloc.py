"""disco_b200_prismatic_noalloc, the matter step for callers that cannot let
the library allocate device memory: the caller passes device inputs and
outputs, the library's scratch is a fixed array inside it.  Its device
outputs must equal those of disco_b200_prismatic (the allocating entry point)
bit for bit, on two calls in a row (the second call finds the first call's
scratch contents and must not depend on them).  Named so that pytest collects
it last; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from disco_b200 import _capi as C
from disco_b200 import prismatic as P
from disco_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _noalloc(lib, torch, w, slab_cap, copy_cap, stream):
    n = w.n
    dev = "cuda"
    pos = torch.tensor(np.stack([w.x, w.y, w.z]), dtype=torch.float64, device=dev)
    out = torch.full((3, n), np.nan, dtype=torch.float64, device=dev)
    new_index = torch.full((n,), -7, dtype=torch.int32, device=dev)
    slab_atoms = torch.full((slab_cap,), -7, dtype=torch.int32, device=dev)
    slab_side = torch.zeros((slab_cap,), dtype=torch.int8, device=dev)
    copies = torch.zeros((copy_cap, 4), dtype=torch.float64, device=dev)   # 32-byte disco_copy
    nl = len(w.slab_loops)
    loops = (C.DiscoSlabLoop * nl)(*w.slab_loops)
    info = (C.DiscoSlabInfo * nl)()
    counts = (ctypes.c_int64 * 3)()
    box = (ctypes.c_double * 3)(*w.box)
    st = lib.disco_b200_prismatic_noalloc(
        pos[0].data_ptr(), pos[1].data_ptr(), pos[2].data_ptr(), n, loops, nl, box,
        out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), new_index.data_ptr(), info,
        slab_atoms.data_ptr(), slab_side.data_ptr(), slab_cap, copies.data_ptr(), copy_cap, counts,
        ctypes.c_void_p(stream))
    return st, counts, info, out, new_index, slab_atoms, slab_side, copies


def test_noalloc_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    lib = C.cuda_lib()
    w = W.bcc_prismatic(cells=40, rmin=10.0, rmax=30.0)          # 128 000 atoms, 16 loops
    ref = P.prismatic(w.x, w.y, w.z, w.slab_loops, w.box)
    k, ns, nc = len(ref["survivors"][0]), len(ref["slab_atoms"]), len(ref["copy_atom"])
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        st, counts, info, out, new_index, slab_atoms, slab_side, copies = _noalloc(
            lib, torch, w, ns + 100, nc + 100, stream)
        torch.cuda.synchronize()
        assert st == C.DISCO_OK, lib.disco_b200_last_error()
        assert list(counts) == [k, ns, nc]
        o = out.cpu().numpy()
        for d in range(3):
            assert np.array_equal(o[d, :k], ref["survivors"][d])
        assert np.array_equal(new_index.cpu().numpy(), ref["new_index"])
        assert np.array_equal(slab_atoms.cpu().numpy()[:ns], ref["slab_atoms"])
        assert np.array_equal(slab_side.cpu().numpy()[:ns], ref["slab_side"])
        cp = copies.cpu().numpy()[:nc]
        assert np.array_equal(cp[:, 0].view(np.int64) & 0xFFFFFFFF, ref["copy_atom"].astype(np.int64))
        assert np.array_equal(cp[:, 1:], ref["copy_shift"])
        got_info = [(info[l].type, info[l].planes, info[l].height, info[l].spacing, tuple(info[l].b[:]),
                     info[l].offset, info[l].count) for l in range(len(w.slab_loops))]
        assert got_info == ref["info"]


def test_noalloc_rejects_sizes_beyond_its_array():
    torch = pytest.importorskip("torch")
    lib = C.cuda_lib()
    w = W.bcc_prismatic(cells=6, rmin=3.0, rmax=5.0, n_inter=1, n_vac=1)
    nl = len(w.slab_loops)
    loops = (C.DiscoSlabLoop * nl)(*w.slab_loops)
    info = (C.DiscoSlabInfo * nl)()
    counts = (ctypes.c_int64 * 3)()
    box = (ctypes.c_double * 3)(*w.box)
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    st = lib.disco_b200_prismatic_noalloc(p, p, p, (1 << 24) + 1, loops, nl, box, p, p, p, p, info,
                                          p, p, 0, None, 0, counts, None)
    assert st == C.DISCO_ELIMIT
    assert b"16777216" in lib.disco_b200_last_error()
    # too small a slab capacity: DISCO_ELIMIT with the size needed in counts[1]
    st, counts, *_ = _noalloc(lib, torch, w, 1, 1, torch.cuda.current_stream().cuda_stream)
    assert st == C.DISCO_ELIMIT and counts[1] > 1


def test_noalloc_copy_capacity_too_small():
    """Enough room for the slabs, room for one copy: DISCO_ELIMIT with the
    number of copies needed in counts[2], the first copy written exactly and
    nothing written past the capacity."""
    torch = pytest.importorskip("torch")
    lib = C.cuda_lib()
    w = W.bcc_prismatic(cells=24, rmin=6.0, rmax=14.0)
    ref = P.prismatic(w.x, w.y, w.z, w.slab_loops, w.box)
    ns, nc = len(ref["slab_atoms"]), len(ref["copy_atom"])
    assert nc > 1
    n = w.n
    pos = torch.tensor(np.stack([w.x, w.y, w.z]), dtype=torch.float64, device="cuda")
    out = torch.empty((3, n), dtype=torch.float64, device="cuda")
    new_index = torch.empty(n, dtype=torch.int32, device="cuda")
    slab_atoms = torch.empty(ns + 100, dtype=torch.int32, device="cuda")
    slab_side = torch.empty(ns + 100, dtype=torch.int8, device="cuda")
    copies = torch.full((4, 4), 7.0, dtype=torch.float64, device="cuda")      # 4 entries, capacity 1
    nl = len(w.slab_loops)
    loops = (C.DiscoSlabLoop * nl)(*w.slab_loops)
    info = (C.DiscoSlabInfo * nl)()
    counts = (ctypes.c_int64 * 3)()
    box = (ctypes.c_double * 3)(*w.box)
    st = lib.disco_b200_prismatic_noalloc(
        pos[0].data_ptr(), pos[1].data_ptr(), pos[2].data_ptr(), n, loops, nl, box,
        out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), new_index.data_ptr(), info,
        slab_atoms.data_ptr(), slab_side.data_ptr(), ns + 100, copies.data_ptr(), 1, counts,
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert st == C.DISCO_ELIMIT
    assert counts[2] == nc and counts[1] == ns
    cp = copies.cpu().numpy()
    assert int(cp[0:1, 0].view(np.int64)[0] & 0xFFFFFFFF) == int(ref["copy_atom"][0])
    assert np.array_equal(cp[0, 1:], ref["copy_shift"][0])
    assert (cp[1:] == 7.0).all()
