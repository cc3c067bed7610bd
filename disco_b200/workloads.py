"""Seeded synthetic workloads of the displacement hot path.

The reference's benchmarks are input files, not datasets; these builders make
the same kind of input (lattice sites in generateLattice order, loop centres
snapped to mid-planes, polylines and loopon grids from the loop class) with
the shapes, sizes and distributions of each workload, from a numpy PCG64
generator with a fixed seed.  Both the GPU path and the CPU oracle consume the
arrays built here, so parity never depends on regenerating an input.

  quadrupole        BCC a0 2.855, 40^3 cells (128 000 atoms), 4 circular glide
                    loops R 30 A on {110}, b = a0/2<111> with alternating
                    signs, centres at the quarter points, 64 chords each
                    (Segment_tolerance 0.0365), nu 0.29, images +-1, line method
  fcc_random        FCC a0 3.615, 150^3 cells (13.5 M atoms), 64 glide loops on
                    random {111} with b = a0/2<110> in the plane: 32 circles R
                    U(10, 40) of 48 chords, 16 hexagons circumradius U(15, 35),
                    16 rectangles with sides U(20, 60); nu 0.34, images +-2
  bcc_prismatic     BCC a0 3.165, 60^3 cells (432 000 atoms), 16 prismatic
                    circles R U(20, 50) on {111} with b = a0/2<111> along n
                    (8 interstitial, 8 vacancy), loopons on a 1 A grid, nu 0.28,
                    images +-1, plus the slab loops of the matter step
"""
from dataclasses import dataclass, field

import numpy as np

from . import geometry as _G

# {111} normals and the <110> directions in each of those planes
_N111 = [(1, 1, 1), (-1, 1, 1), (1, -1, 1), (1, 1, -1)]
_D110 = [(1, -1, 0), (1, 0, -1), (0, 1, -1), (1, 1, 0), (1, 0, 1), (0, 1, 1)]


def _in_plane_110(n):
    out = []
    for d in _D110:
        if d[0] * n[0] + d[1] * n[1] + d[2] * n[2] == 0:
            out += [d, tuple(-t for t in d)]
    return out


@dataclass
class Workload:
    name: str
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    loops: list
    box: tuple
    images: int
    nu: float
    method: str                      # "line" or "loopons"
    lattice: int = _G.BCC
    a0: float = 0.0
    cells: tuple = (0, 0, 0)
    slab_loops: list = field(default_factory=list)
    geom: list = field(default_factory=list)

    @property
    def n(self):
        return int(self.x.shape[0])

    def evals_per_atom(self):
        """(segments or loopons) x images, summed over the loops."""
        k = sum(len(lp.vx) if lp.line else len(lp.x) for lp in self.loops)
        return k * (2 * self.images + 1) ** 3

    def subset(self, idx):
        """The same loops and box over a subset of the atoms (sampling)."""
        w = Workload(**{**self.__dict__})
        w.x, w.y, w.z = self.x[idx].copy(), self.y[idx].copy(), self.z[idx].copy()
        w.name = self.name + f"[{len(idx)} atoms]"
        return w


def quadrupole(cells=40, a0=2.855, radius=30.0, eps=0.0365, nu=0.29, images=1, da=1.0, geom=None):
    """Four circular shear loops forming a quadrupole (the pattern of the
    reference's Examples/quadrupole_circle.yaml), line method."""
    G = geom or _G
    L = cells * a0
    q = L / 4.0
    specs = [((-q, -q, 0.0), (1, -1, -1), (1, 1, 0)),
             ((-q, q, 0.0), (-1, -1, 1), (-1, 1, 0)),
             ((q, -q, 0.0), (-1, -1, -1), (-1, 1, 0)),
             ((q, q, 0.0), (1, -1, 1), (1, 1, 0))]
    x, y, z = G.lattice(G.BCC, cells, cells, cells, a0)
    loops, geom = [], []
    for c, m, n in specs:
        cs, _ = G.snap(c, n, a0, cells, cells, cells, G.BCC)
        lp = G.Loop.circle(da, radius, cs, m, n, a0)
        geom.append(lp)
        loops.append(lp.line_data(eps))
    return Workload("quadrupole", x, y, z, loops, (L, L, L), images, nu, "line", G.BCC, a0,
                    (cells, cells, cells), geom=geom)


def _fcc_glide_loop(rng, kind, cells, a0, da, chords, G):
    """One glide loop of the fcc_random distribution: a random {111} plane, b =
    a0/2<110> in it, centre uniform in the box (snapped to a mid-plane)."""
    L = cells * a0
    n = _N111[rng.integers(len(_N111))]
    ms = _in_plane_110(n)
    m = ms[rng.integers(len(ms))]
    c = rng.uniform(-L / 2, L / 2, size=3)
    cs, _ = G.snap(c, n, a0, cells, cells, cells, G.FCC)
    if kind == "circle":
        R = rng.uniform(10.0, 40.0)
        lp = G.Loop.circle(da, R, cs, m, n, a0)
        P = lp.polyline(G.circle_eps_for_chords(R, chords))
    elif kind == "hexagon":
        R = rng.uniform(15.0, 35.0)
        lp = G.Loop.polygon(da, G.regular_polygon(6, R, m, n), 0.0, cs, m, n, a0)
        P = lp.polyline(0.01)
    else:
        s1, s2 = rng.uniform(20.0, 60.0, size=2)
        lp = G.Loop.rectangle(da, s1 / 2, s2 / 2, 0.0, cs, m, n, a0)
        P = lp.polyline(0.01)
    return lp, lp.line_data(vertices=P)


def fcc_random(cells=150, a0=3.615, nu=0.34, images=2, seed=2, n_circles=32, n_hex=16, n_rect=16,
               chords=48, da=1.0, geom=None):
    """64 random shear loops in an FCC box, line method."""
    G = geom or _G
    rng = np.random.default_rng(seed)
    L = cells * a0
    x, y, z = G.lattice(G.FCC, cells, cells, cells, a0)
    loops, geom = [], []
    kinds = ["circle"] * n_circles + ["hexagon"] * n_hex + ["rectangle"] * n_rect
    for kind in kinds:
        lp, ld = _fcc_glide_loop(rng, kind, cells, a0, da, chords, G)
        geom.append(lp)
        loops.append(ld)
    return Workload("fcc_random", x, y, z, loops, (L, L, L), images, nu, "line", G.FCC, a0,
                    (cells, cells, cells), geom=geom)


def fcc_random_loops(count, seed, cells=150, a0=3.615, chords=48, da=1.0, geom=None):
    """`count` loops drawn from the fcc_random distribution (kinds in its
    proportions: half circles, a quarter hexagons, a quarter rectangles)."""
    rng = np.random.default_rng(seed)
    kinds = rng.choice(["circle", "circle", "hexagon", "rectangle"], size=count)
    return [_fcc_glide_loop(rng, k, cells, a0, da, chords, geom or _G)[1] for k in kinds]


def bcc_prismatic(cells=60, a0=3.165, nu=0.28, images=1, seed=3, n_inter=8, n_vac=8, da=1.0,
                  rmin=20.0, rmax=50.0, geom=None):
    """16 prismatic circular loops (loopon method) with their slab loops."""
    G = geom or _G
    rng = np.random.default_rng(seed)
    L = cells * a0
    x, y, z = G.lattice(G.BCC, cells, cells, cells, a0)
    kinds = np.array(["inter"] * n_inter + ["vac"] * n_vac)
    rng.shuffle(kinds)
    loops, geom, slabs = [], [], []
    for kind in kinds:
        n = _N111[rng.integers(len(_N111))]
        m = n if kind == "vac" else tuple(-t for t in n)      # m.n > 0: vacancy
        R = rng.uniform(rmin, rmax)
        c = rng.uniform(-L / 2, L / 2, size=3)
        cs, d = G.snap(c, n, a0, cells, cells, cells, G.BCC)
        lp = G.Loop.circle(da, R, cs, m, n, a0)
        geom.append(lp)
        loops.append(lp.loopon_data())
        slabs.append(lp.slab_loop(d, apply=True, frank=False, a0=a0))
    return Workload("bcc_prismatic", x, y, z, loops, (L, L, L), images, nu, "loopons", G.BCC, a0,
                    (cells, cells, cells), slab_loops=slabs, geom=geom)


def on_plane(cells=12, a0=2.855, nu=0.35, images=1, radius=8.8, eps=0.0365, geom=None):
    """Loops whose planes pass through lattice sites: each centre is an atom
    (not snapped to a mid-plane), so every loop has atoms exactly on its plane
    inside and outside the contour, one at its centre, and some on the rays
    from the centre to its vertices.  BCC box, line method; circles on (001),
    (110), (1-10), (111) and (112), a hexagon on (1-10), a rectangle on (001).
    The reference's cut surface decides which side such an atom is on by the
    rounding of its solid-angle arithmetic (Code/barnett.hpp:69-72)."""
    G = geom or _G
    L = cells * a0
    x, y, z = G.lattice(G.BCC, cells, cells, cells, a0)
    q = L / 4.0
    specs = [("circle", (0, 0, 1), (1, 0, 0), (-q, -q, -q)),
             ("circle", (1, 1, 0), (1, -1, 1), (q, -q, -q)),
             ("circle", (1, -1, 0), (1, 1, 1), (-q, q, -q)),
             ("circle", (1, 1, 1), (1, 1, 1), (q, q, -q)),
             ("circle", (1, 1, 2), (1, 1, -1), (-q, -q, q)),
             ("hexagon", (1, -1, 0), (1, 1, -1), (q, -q, q)),
             ("rectangle", (0, 0, 1), (0, 1, 0), (-q, q, q))]
    pos = np.stack([x, y, z], 1)
    loops, geom = [], []
    for kind, n, m, target in specs:
        i = int(np.argmin(((pos - np.array(target)) ** 2).sum(1)))
        c = (float(x[i]), float(y[i]), float(z[i]))
        if kind == "circle":
            lp = G.Loop.circle(1.0, radius, c, m, n, a0)
            P = lp.polyline(eps)
        elif kind == "hexagon":
            lp = G.Loop.polygon(1.0, G.regular_polygon(6, radius, m, n), 0.0, c, m, n, a0)
            P = lp.polyline(0.01)
        else:
            lp = G.Loop.rectangle(1.0, radius, 0.6 * radius, 0.0, c, m, n, a0)
            P = lp.polyline(0.01)
        geom.append(lp)
        loops.append(lp.line_data(vertices=P))
    return Workload("on_plane", x, y, z, loops, (L, L, L), images, nu, "line", G.BCC, a0,
                    (cells, cells, cells), geom=geom)


_N110 = [(1, 1, 0), (1, -1, 0), (1, 0, 1), (1, 0, -1), (0, 1, 1), (0, 1, -1)]
_N112 = [(1, 1, 2), (1, 1, -2), (1, -1, 2), (-1, 1, 2), (1, 2, 1), (1, 2, -1), (1, -2, 1), (-1, 2, 1),
         (2, 1, 1), (2, 1, -1), (2, -1, 1), (-2, 1, 1)]
_B111 = [(1, 1, 1), (1, 1, -1), (1, -1, 1), (-1, 1, 1)]


def batch(nsamples=256, a0=2.855, edge=(20, 80), nloops=(1, 32), radius=(8.0, 40.0),
          segments=(16, 128), images=(1, 3), nu=0.29, seed=4, da=1.0, geom=None):
    """Many independent BCC samples for the batched form: box edges uniform
    integers in `edge` (cells, independent per axis), 1-32 glide loops each
    (circles of `segments` chords or regular hexagons, radius in `radius`), on
    random {110}<111> or {112}<111> systems with a random sign of b, centres
    uniform, images +-U{images}."""
    G = geom or _G
    rng = np.random.default_rng(seed)
    out = []
    for s in range(nsamples):
        nx, ny, nz = (int(v) for v in rng.integers(edge[0], edge[1] + 1, size=3))
        L = (nx * a0, ny * a0, nz * a0)
        x, y, z = G.lattice(G.BCC, nx, ny, nz, a0)
        loops, geom = [], []
        for _ in range(int(rng.integers(nloops[0], nloops[1] + 1))):
            fam = _N110 if rng.random() < 0.5 else _N112
            n = fam[rng.integers(len(fam))]
            bs = [b for b in _B111 if b[0] * n[0] + b[1] * n[1] + b[2] * n[2] == 0]
            m = bs[rng.integers(len(bs))]
            if rng.random() < 0.5:
                m = tuple(-t for t in m)
            c = np.array([rng.uniform(-l / 2, l / 2) for l in L])
            cs, _ = G.snap(c, n, a0, nx, ny, nz, G.BCC)
            R = rng.uniform(*radius)
            if rng.random() < 0.5:
                k = int(rng.integers(segments[0], segments[1] + 1))
                lp = G.Loop.circle(da, R, cs, m, n, a0)
                P = lp.polyline(G.circle_eps_for_chords(R, k))
            else:
                lp = G.Loop.polygon(da, G.regular_polygon(6, R, m, n), 0.0, cs, m, n, a0)
                P = lp.polyline(0.01)
            geom.append(lp)
            loops.append(lp.line_data(vertices=P))
        im = int(rng.integers(images[0], images[1] + 1))
        out.append(Workload(f"batch[{s}]", x, y, z, loops, L, im, nu, "line", G.BCC, a0, (nx, ny, nz),
                            geom=geom))
    return out


# Full-size workloads by name (bench and tests select them by these names).
FULL = {
    "quadrupole": quadrupole,
    "fcc_random": fcc_random,
    "bcc_prismatic": bcc_prismatic,
}
