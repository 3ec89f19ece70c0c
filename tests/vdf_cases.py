"""Seeded meshes and sample points for PSI.VDF and PSI.RStarTree.

Lattices with a mild displacement (the sheet stays single-stream almost
everywhere) and a strong one (several streams per point), periodic and open,
with at most 32 elements (the reference's tree is one leaf: its results come
in descending element order) and with more (the same set in another order)."""
from __future__ import annotations

import numpy as np

import oracle as O
from ann_cases import lattice

CASES = {
    # name: (particles per side, displacement amplitude in box units, periodic, max level, tolerance)
    "open4_mild": (4, 0.03, False, 0, 1.0),
    "open4_strong": (4, 0.25, False, 1, 0.02),
    "periodic3_mild": (3, 0.04, True, 0, 1.0),
    "periodic3_refined": (3, 0.08, True, 2, 0.01),
    "open7_strong": (7, 0.2, False, 0, 1.0),
    "periodic5": (5, 0.1, True, 1, 0.02),
}
SMALL = [k for k, v in CASES.items() if (v[0] if v[2] else v[0] - 1) ** 3 <= 32]
LARGE = [k for k in CASES if k not in SMALL]


def make(name):
    n, amp, periodic, lvl, tol = CASES[name]
    pos, conn = lattice(n, 1.0, amp, periodic, 11 + n)
    rng = np.random.default_rng(n)
    vel = rng.normal(size=pos.shape)
    mass = rng.uniform(0.5, 1.5, conn.shape[0])
    box = ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)) if periodic else None
    pts = np.random.default_rng(100 + n).uniform(0.05, 0.95, (12, 3))
    pts[0] = (0.0, 0.0, 0.0)  # the origin: the open mesh's default window is the zero box
    return dict(pos=pos, conn=conn, vel=vel, mass=mass, periodic_box=box, maxlvl=lvl, reftol=tol, points=pts)


def vdf(c, kind, point, tree):
    window = O.tree_window(c["periodic_box"]) if tree else None
    return O.sample_vdf(kind, c["pos"], c["conn"], point, vel=c["vel"], mass=c["mass"], periodic_box=c["periodic_box"],
                        window=window, reftol=c["reftol"], maxlvl=c["maxlvl"])


def sorted_samples(rho, vel):
    a = np.column_stack([rho, vel])
    return a[np.lexsort(a.T[::-1])] if len(a) else a
