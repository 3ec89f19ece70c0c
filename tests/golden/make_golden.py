"""Generate tests/golden/golden.npz from the reference implementation.

    python tests/golden/make_golden.py

Runs PyPSI's own density path (its C sources compiled unchanged into
oracle/_ref/libpsiref.so by oracle/Makefile) on small seeded inputs and stores
inputs, arguments and output fields.  The reference publishes no per-voxel
vectors of its own (its only known answers are the tutorial's global mass
errors), so these fixtures carry its behaviour to machines where the
reference sources are absent.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

import oracle as O  # noqa: E402
from pypsi_b200.synth import zeldovich  # noqa: E402

BOX = ((0.0, 0.0, 0.0), (100.0, 100.0, 100.0))


def cases():
    pos, vel = zeldovich(4, 2.0, 201)
    yield "g_c2", dict(pos=pos.reshape(-1, 3), vel=vel.reshape(-1, 3), conn=O.block_connectivity((4, 4, 4), True),
                       mass=None, periodic_box=BOX, n=(8, 8, 8), bounds=BOX, fields=["x", "v", "xx", "xv", "vv"],
                       reftol=1.0, maxlvl=0)
    pos, vel = zeldovich(4, 2.0, 202)
    yield "g_refine", dict(pos=pos.reshape(-1, 3), vel=vel.reshape(-1, 3), conn=O.block_connectivity((4, 4, 4), True),
                           mass=None, periodic_box=BOX, n=(8, 8, 8), bounds=BOX, fields=["v"], reftol=0.2, maxlvl=2)
    pos, vel = zeldovich(6, 1.0, 203)
    yield "g_sub", dict(pos=pos.reshape(-1, 3), vel=vel.reshape(-1, 3), conn=O.block_connectivity((6, 6, 6), True),
                        mass=None, periodic_box=BOX, n=(6, 5, 7), bounds=((10.0, -5.0, 20.0), (60.0, 40.0, 95.0)),
                        fields=["x", "v", "xx", "vv"], reftol=1.0, maxlvl=0)
    rng = np.random.default_rng(204)
    nt = 20
    p = (rng.uniform(0.15, 0.85, (nt, 1, 3)) + rng.normal(0, 0.08, (nt, 4, 3))).reshape(-1, 3)
    yield "g_tets", dict(pos=p, vel=rng.normal(size=p.shape), conn=np.arange(4 * nt, dtype=np.int32).reshape(nt, 4),
                         mass=rng.uniform(0.5, 1.5, nt), periodic_box=None, n=(8, 8, 8),
                         bounds=((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)), fields=["x", "v", "xx", "xv", "vv"], reftol=1.0,
                         maxlvl=0)


def main():
    O.build()
    data = {}
    meta = {}
    for name, c in cases():
        out = O.voxelize("reference", **c)
        for k in ("pos", "vel", "conn"):
            data[f"{name}/in_{k}"] = c[k]
        if c["mass"] is not None:
            data[f"{name}/in_mass"] = c["mass"]
        for f, a in out.items():
            data[f"{name}/out_{f}"] = a
        meta[name] = {k: c[k] for k in ("periodic_box", "n", "bounds", "fields", "reftol", "maxlvl")}
        meta[name]["has_mass"] = c["mass"] is not None
    data["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **data)
    print("wrote", os.path.join(HERE, "golden.npz"), sorted(meta))


if __name__ == "__main__":
    main()
