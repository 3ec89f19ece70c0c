"""Synthetic Gadget-2 (format 1) snapshots for the loader tests.

A seeded particle lattice of n^3 particles in a periodic box, displaced by a
few smooth sine modes (a Zel'dovich-like field, so the trilinear elements shear
and overlap as a late snapshot's do), wrapped into [0, box), with velocities
proportional to the displacement, written in a random particle order with their
lattice indices as IDs.  'gevolution' files use 64-bit IDs numbered in 4^3
tiles: the lattice point of ID t*64+s is the tile t's origin plus the slot s
position of the tile numbering."""
from __future__ import annotations

import struct

import numpy as np


def lattice_particles(n: int, box: float, amp: float = 0.3, seed: int = 0):
    """Positions (n^3, 3) and velocities of the row-major lattice (i, j, k)."""
    rng = np.random.default_rng(seed)
    q = (np.stack(np.meshgrid(*(np.arange(n),) * 3, indexing="ij"), axis=-1).reshape(-1, 3) + 0.5) * (box / n)
    disp = np.zeros_like(q)
    for _ in range(4):
        k = rng.integers(1, 3, size=3) * rng.choice([-1, 1], size=3)
        a = rng.normal(size=3) * amp * box / n
        ph = rng.uniform(0, 2 * np.pi)
        disp += a * np.sin(2 * np.pi * (q @ k) / box + ph)[:, None]
    pos = np.mod(q + disp, box)
    vel = 10.0 * disp + rng.normal(scale=0.01, size=disp.shape)
    return pos, vel


def write_snapshot(path: str, pos_rows, vel_rows, mass1: float, box: float, flavour: str = "gadget2", seed: int = 0,
                   ids=None, header_npart=None):
    """Write particles whose row r belongs to ID r, in a shuffled file order.
    `ids` overrides the ID block (for malformed files)."""
    rng = np.random.default_rng(seed + 1)
    npart = pos_rows.shape[0]
    order = rng.permutation(npart)
    file_ids = order if ids is None else np.asarray(ids)
    idt = np.int32 if flavour == "gadget2" else np.int64
    hdr = bytearray(256)
    npart6 = [0, npart if header_npart is None else header_npart, 0, 0, 0, 0]
    struct.pack_into("<6i", hdr, 0, *npart6)
    struct.pack_into("<6d", hdr, 24, 0.0, mass1, 0.0, 0.0, 0.0, 0.0)
    struct.pack_into("<dd", hdr, 72, 1.0, 0.0)  # scale factor, redshift
    struct.pack_into("<6I", hdr, 96, *npart6)
    struct.pack_into("<i", hdr, 124, 1)  # num_files
    struct.pack_into("<4d", hdr, 128, box, 0.3, 0.7, 0.7)

    def block(b: bytes) -> bytes:
        m = struct.pack("<I", len(b) & 0xFFFFFFFF)
        return m + b + m

    with open(path, "wb") as f:
        f.write(block(bytes(hdr)))
        f.write(block(np.asarray(pos_rows, np.float32)[order].tobytes()))
        f.write(block(np.asarray(vel_rows, np.float32)[order].tobytes()))
        f.write(block(file_ids.astype(idt).tobytes()))


def gevolution_rows(n: int):
    """Lattice index (row-major, i slowest) of every gevolution ID 0..n^3-1."""
    import oracle as O

    to_cube, _ = O._gevolution_tile_tables()
    tn = n // 4
    p = np.arange(n ** 3)
    t = p // 64
    tile = np.stack([t % tn, (t // tn) % tn, t // (tn * tn)], axis=1)
    ijk = 4 * tile + to_cube[p % 64]
    return (ijk[:, 0] * n + ijk[:, 1]) * n + ijk[:, 2]


def make_snapshot(path: str, n: int, box: float = 40.0, mass1: float = 15.0, flavour: str = "gadget2", seed: int = 0):
    """A synthetic snapshot of n^3 particles; returns (pos, vel) by ID."""
    pos, vel = lattice_particles(n, box, seed=seed)
    if flavour == "gevolution":
        rows = gevolution_rows(n)
        pos, vel = pos[rows], vel[rows]
    write_snapshot(path, pos, vel, mass1, box, flavour, seed=seed)
    return pos, vel
