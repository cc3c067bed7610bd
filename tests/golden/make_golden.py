"""Generates tests/golden/reference_vectors.npz from the reference's OWN code.

Run where the reference tree exists (it is compiled in place into
oracle/_ref by oracle/build_oracle.py):  python tests/golden/make_golden.py

Every array in the file is either an input (atoms, polylines, loopons, slab
loops) or the output of a reference function on that input:
  line_*      kroupaCPU line branch (Code/backend_cpu.cpp:40-63), quadrupole of
              4 circular glide loops in a 10^3-cell BCC box, nu 0.35, images +-1
  loopon_*    kroupaCPU loopon branch (Code/backend_cpu.cpp:64-96), 16 prismatic
              circles in a 10^3-cell BCC box
  plane_*     kroupaCPU line branch on loops whose planes pass through lattice
              sites (workloads.on_plane: atoms exactly on a loop's plane,
              inside and outside the contour, at its centre and on fan edges),
              nu 0.35, images +-1
  slab_*      prismaticSlab (Code/prismatic.cpp:36-74) driven as
              Code/main.cpp:586-687 drives it, 16 prismatic circles, 12^3 cells
Outputs are stored for both builds of the reference (default flags and
-ffp-contract=off).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "reference_vectors.npz")


def _loops_arrays(loops, prefix, d):
    d[prefix + "_nv"] = np.array([len(l.vx) if l.line else len(l.x) for l in loops], dtype=np.int32)
    if loops[0].line:
        d[prefix + "_V"] = np.concatenate([np.stack([l.vx, l.vy, l.vz], 1) for l in loops])
        d[prefix + "_c"] = np.array([[l.cx, l.cy, l.cz] for l in loops])
    else:
        d[prefix + "_P"] = np.concatenate([np.stack([l.x, l.y, l.z], 1) for l in loops])
    d[prefix + "_phys"] = np.array([[l.phys.bx, l.phys.by, l.phys.bz, l.phys.mx, l.phys.my, l.phys.mz,
                                     l.phys.nx, l.phys.ny, l.phys.nz, l.phys.dS] for l in loops])


def main():
    from oracle import build_oracle
    import __graft_entry__ as G
    build_oracle.build(verbose=False, reference=G.REFERENCE_CODE)
    import oracle as O
    from disco_b200 import workloads as W
    from disco_b200 import _capi as C
    if not O.have_ref():
        raise SystemExit("the reference tree is needed to make the golden vectors")
    d = {}
    w = W.quadrupole(cells=10, radius=8.0, eps=0.0365)
    d["line_box"] = np.array(w.box)
    d["line_xyz"] = np.stack([w.x, w.y, w.z], 1)
    _loops_arrays(w.loops, "line", d)
    d["line_u"] = np.stack(O.ref_displace(w.x, w.y, w.z, w.loops, w.box), 1)
    d["line_u_nofma"] = np.stack(O.ref_displace(w.x, w.y, w.z, w.loops, w.box, nofma=True), 1)

    w = W.bcc_prismatic(cells=10, rmin=4.0, rmax=8.0)
    d["loopon_box"] = np.array(w.box)
    d["loopon_xyz"] = np.stack([w.x, w.y, w.z], 1)
    _loops_arrays(w.loops, "loopon", d)
    d["loopon_u"] = np.stack(O.ref_displace(w.x, w.y, w.z, w.loops, w.box), 1)
    d["loopon_u_nofma"] = np.stack(O.ref_displace(w.x, w.y, w.z, w.loops, w.box, nofma=True), 1)

    w = W.on_plane()
    d["plane_box"] = np.array(w.box)
    d["plane_xyz"] = np.stack([w.x, w.y, w.z], 1)
    _loops_arrays(w.loops, "plane", d)
    d["plane_u"] = np.stack(O.ref_displace(w.x, w.y, w.z, w.loops, w.box), 1)
    d["plane_u_nofma"] = np.stack(O.ref_displace(w.x, w.y, w.z, w.loops, w.box, nofma=True), 1)

    w = W.bcc_prismatic(cells=12, rmin=4.0, rmax=9.0, seed=33)
    refl = [O.RefLoop(0, 1.0, g.center, g.m_in, g.n_in, w.a0, radius=g.g.radius)
            for g in w.geom]
    spacing = [s.spacing for s in w.slab_loops]
    r = O.ref_prismatic(refl, spacing, w.x, w.y, w.z, w.box)
    d["slab_box"] = np.array(w.box)
    d["slab_xyz"] = np.stack([w.x, w.y, w.z], 1)
    d["slab_loops"] = np.frombuffer(bytes((C.DiscoSlabLoop * len(w.slab_loops))(*w.slab_loops)),
                                    dtype=np.uint8)
    d["slab_atoms"] = r["slab_atoms"]
    d["slab_side"] = r["slab_side"]
    d["slab_new_index"] = r["new_index"]
    d["slab_counts"] = np.array([len(r["survivors"][0]), len(r["slab_atoms"]), len(r["copy_atom"])])
    d["slab_info"] = np.array([[i[0], i[1], i[2], i[3], *i[4], i[5], i[6]] for i in r["info"]])
    d["slab_copy_atom"] = r["copy_atom"]
    d["slab_copy_shift"] = r["copy_shift"]
    np.savez_compressed(OUT, **d)
    print(f"wrote {OUT}: " + ", ".join(f"{k}{tuple(v.shape)}" for k, v in d.items()))


if __name__ == "__main__":
    main()
