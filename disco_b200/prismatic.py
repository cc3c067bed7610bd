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
