"""Prismatic matter step and output epilogue on the GPU (C-ABI wrappers).

prismatic(): prismaticSlab (Code/prismatic.cpp:36-74) for every loop with
b.n != 0, driven as Code/main.cpp:586-687 drives it: vacancy slabs removed,
interstitial slabs copied, survivors compacted in order, copies of removed
atoms dropped.  finalize(): copies appended with u(source) + shift, positions
r = x + u wrapped once and shifted by +L/2 (Code/main.cpp:733-743, 797-818).
"""
import ctypes

import numpy as np

from . import _capi as C


def _box(box):
    return (ctypes.c_double * 3)(*[float(v) for v in box])


def prismatic(x, y, z, slab_loops, box):
    """Returns a dict: survivors (x, y, z), new_index, info (per loop: type,
    planes, height, spacing, b, offset, count), slab_atoms, slab_side,
    copy_atom (renumbered sources), copy_shift."""
    lib = C.cuda_lib()
    n = len(x)
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    nl = len(slab_loops)
    arr = (C.DiscoSlabLoop * max(1, nl))(*slab_loops)
    xo, yo, zo = np.empty(max(1, n)), np.empty(max(1, n)), np.empty(max(1, n))
    new_index = np.empty(max(1, n), dtype=np.int32)
    info = (C.DiscoSlabInfo * max(1, nl))()
    counts = (ctypes.c_int64 * 3)()
    cap_s, cap_c = 1 << 14, 1 << 14
    while True:
        slab_atoms = np.empty(cap_s, dtype=np.int32)
        slab_side = np.empty(cap_s, dtype=np.int8)
        copies = (C.DiscoCopy * cap_c)()
        st = lib.disco_b200_prismatic(x.ctypes.data, y.ctypes.data, z.ctypes.data, n, arr, nl, _box(box),
                                      xo.ctypes.data, yo.ctypes.data, zo.ctypes.data,
                                      new_index.ctypes.data, info, slab_atoms.ctypes.data,
                                      slab_side.ctypes.data, cap_s, copies, cap_c, counts)
        if st == C.DISCO_ELIMIT and (counts[1] > cap_s or counts[2] > cap_c):
            cap_s, cap_c = max(cap_s, counts[1]), max(cap_c, counts[2])
            continue
        C.check(st, lib)
        break
    k, ns, nc = counts[0], counts[1], counts[2]
    cp = np.frombuffer(bytes(copies), dtype=np.dtype([("atom", np.int32), ("r", np.int32),
                                                       ("shift", np.float64, 3)]), count=nc)
    return {
        "survivors": (xo[:k].copy(), yo[:k].copy(), zo[:k].copy()),
        "new_index": new_index[:n].copy(),
        "info": [(info[l].type, info[l].planes, info[l].height, info[l].spacing, tuple(info[l].b[:]),
                  info[l].offset, info[l].count) for l in range(nl)],
        "slab_atoms": slab_atoms[:ns].copy(),
        "slab_side": slab_side[:ns].copy(),
        "copy_atom": cp["atom"].copy(),
        "copy_shift": cp["shift"].copy(),
    }


def finalize(x, y, z, ux, uy, uz, copy_atom, copy_shift, box):
    """(fx, fy, fz, ux, uy, uz) of the n atoms followed by the copies."""
    lib = C.cuda_lib()
    n, nc = len(x), len(copy_atom)
    cps = (C.DiscoCopy * max(1, nc))()
    for i in range(nc):
        cps[i].atom = int(copy_atom[i])
        cps[i].shift = C.D3(*copy_shift[i])
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, ux, uy, uz)]
    out = [np.empty(max(1, n + nc)) for _ in range(6)]
    C.check(lib.disco_b200_finalize(*[a.ctypes.data for a in arrs], n, cps, nc, _box(box),
                                    *[o.ctypes.data for o in out]), lib)
    return [o[:n + nc] for o in out]


def _main():
    """python -m disco_b200.prismatic [--cells N] [--reps R]: the matter step
    (disco_b200_prismatic_noalloc) on device arrays, BCC N^3 cells with the 16
    loops of the bcc_prismatic distribution, timed with CUDA events; the case
    the compaction kernels' ncu summaries are taken on."""
    import argparse
    import torch
    from . import workloads as W
    p = argparse.ArgumentParser()
    p.add_argument("--cells", type=int, default=128)
    p.add_argument("--reps", type=int, default=5)
    a = p.parse_args()
    lib = C.cuda_lib()
    w = W.bcc_prismatic(cells=a.cells)
    n = w.n
    pos = torch.tensor(np.stack([w.x, w.y, w.z]), dtype=torch.float64, device="cuda")
    out = torch.empty((3, n), dtype=torch.float64, device="cuda")
    new_index = torch.empty(n, dtype=torch.int32, device="cuda")
    cap = 1 << 21
    slab_atoms = torch.empty(cap, dtype=torch.int32, device="cuda")
    slab_side = torch.empty(cap, dtype=torch.int8, device="cuda")
    copies = torch.empty((cap, 4), dtype=torch.float64, device="cuda")
    nl = len(w.slab_loops)
    sl = (C.DiscoSlabLoop * nl)(*w.slab_loops)
    info = (C.DiscoSlabInfo * nl)()
    counts = (ctypes.c_int64 * 3)()
    s = torch.cuda.current_stream()

    def call():
        C.check(lib.disco_b200_prismatic_noalloc(
            pos[0].data_ptr(), pos[1].data_ptr(), pos[2].data_ptr(), n, sl, nl, _box(w.box),
            out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), new_index.data_ptr(), info,
            slab_atoms.data_ptr(), slab_side.data_ptr(), cap, copies.data_ptr(), cap, counts,
            ctypes.c_void_p(s.cuda_stream)), lib)

    call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        call()
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) * 1e-3 / a.reps
    print(f"matter step: {n} atoms, {counts[0]} survivors, {counts[1]} slab atoms, {counts[2]} copies: "
          f"{t * 1e3:.3f} ms per call, {52.0 * n / t / 1e9:.0f} GB/s of algorithmic bytes (52 B/atom)")


if __name__ == "__main__":
    _main()
