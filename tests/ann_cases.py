"""Seeded meshes for annihilation mode (PSI.voxels(mode='annihilation')).

Every case overlaps itself: trilinear lattices displaced past shell crossing,
periodic ones whose elements straddle the box edge, and random tets.  Cases of
at most 32 kept elements are the ones the reference's R*-tree answers in
plain descending element order (one leaf), so the oracle and the GPU match it
bit for bit there; beyond that only the order of the sums differs."""
from __future__ import annotations

import zlib

import numpy as np

import oracle as O


def lattice(n, L, amp, periodic, seed):
    r = np.random.default_rng(seed)
    q = (np.stack(np.meshgrid(*(np.arange(n),) * 3, indexing="ij"), -1).reshape(-1, 3) + 0.5) * (L / n)
    k = 2 * np.pi / L
    d = amp * np.stack([np.sin(k * q[:, 0] + 1.0) * np.cos(k * q[:, 1]), np.sin(k * q[:, 1] + 2.0),
                        np.cos(k * q[:, 2] + 0.3) * np.sin(k * q[:, 0])], 1)
    d += r.normal(scale=0.05 * L / n, size=d.shape)
    pos = q + d
    if periodic:
        pos = np.mod(pos, L)
    return pos, O.block_connectivity((n, n, n), periodic)


def make(name):
    """dict(n, bounds, pos, conn, mass, periodic_box, reftol, maxlvl)."""
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    unit = ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    c = dict(n=(8, 8, 8), bounds=unit, mass=None, periodic_box=None, reftol=1.0, maxlvl=0)
    if name in ("tets", "degenerate"):
        r = np.random.default_rng(2)
        conn = np.array([r.choice(40, 4, replace=False) for _ in range(10)], dtype=np.int32)
        if name == "degenerate":
            conn[9, 1] = conn[9, 0]  # a tet of zero volume: rho = inf, as in the reference
        c.update(pos=np.random.default_rng(1).uniform(0, 1, (40, 3)), conn=conn,
                 mass=np.random.default_rng(3).uniform(0.5, 2, 10))
    elif name == "block3":
        pos, conn = lattice(3, 1.0, 0.3, False, 2)
        c.update(n=(10, 10, 10), pos=pos, conn=conn)
    elif name == "periodic3":
        pos, conn = lattice(3, 1.0, 0.25, True, 3)
        c.update(pos=pos, conn=conn, periodic_box=unit, mass=rng.uniform(0.5, 1.5, 27))
    elif name == "periodic3_refined":
        pos, conn = lattice(3, 1.0, 0.25, True, 3)
        c.update(pos=pos, conn=conn, periodic_box=unit, maxlvl=1, reftol=0.3)
    elif name == "window3":
        # a window inside the box: window planes cut the tet pairs
        pos, conn = lattice(3, 1.0, 0.3, False, 5)
        c.update(n=(7, 9, 6), bounds=((0.2, 0.15, 0.3), (0.85, 0.9, 0.8)), pos=pos, conn=conn)
    elif name == "periodic5":
        pos, conn = lattice(5, 1.0, 0.3, True, 4)
        c.update(n=(12, 12, 12), bounds=((0.1, 0.0, 0.0), (0.9, 1.0, 1.0)), pos=pos, conn=conn, periodic_box=unit)
    elif name == "block6":
        pos, conn = lattice(6, 2.0, 0.5, False, 6)
        c.update(n=(20, 20, 20), bounds=((0.0, 0.0, 0.0), (2.0, 2.0, 2.0)), pos=pos, conn=conn)
    else:
        raise KeyError(name)
    return c


SMALL = ["tets", "block3", "periodic3", "periodic3_refined", "window3"]  # <= 32 kept elements
LARGE = ["periodic5", "block6"]


def run_oracle(c, kind="restatement", counters=False):
    return O.voxelize(kind, c["n"], c["bounds"], c["pos"], c["conn"], mass=c["mass"], periodic_box=c["periodic_box"],
                      reftol=c["reftol"], maxlvl=c["maxlvl"], counters=counters, mode="annihilation")
