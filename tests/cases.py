"""Seeded parity cases shared by the oracle pins and the GPU parity tests.

Each case is a dict with the grid (n, bounds, fields), the mesh (loader and
arrays) and the voxels() refinement arguments.  Sizes are chosen so that the
CPU oracle finishes each in about a second.
"""
from __future__ import annotations

import numpy as np

from pypsi_b200.synth import lattice, zeldovich

BOX = ((0.0, 0.0, 0.0), (100.0, 100.0, 100.0))
ALL = ["x", "v", "xx", "xv", "vv"]


def _block(pos, vel, n_grid, fields, box=BOX, bounds=None, reftol=1.0, maxlvl=0, mass=None, periodic=True):
    return dict(kind="block", pos=pos, vel=vel, mass=mass, periodic_box=box if periodic else None,
                n=(n_grid,) * 3 if np.isscalar(n_grid) else tuple(n_grid), bounds=bounds or box, fields=list(fields),
                reftol=reftol, maxlvl=maxlvl)


def make(name: str) -> dict:
    if name == "c1_small":  # the 32^3 -> 64^3 density workload's shape at 16^3 particles
        pos, vel = zeldovich(16, 0.3, 101)
        return _block(pos, vel, 32, [])
    if name == "c2_small":  # the 128^3 -> 256^3 workload's shape: shell-crossed, all order-2 fields
        pos, vel = zeldovich(16, 2.0, 102)
        return _block(pos, vel, 32, ALL)
    if name == "c2_order1":
        pos, vel = zeldovich(16, 2.0, 103)
        return _block(pos, vel, 32, ["x", "v"])
    if name == "rms3_vvonly":
        pos, vel = zeldovich(16, 3.0, 104)
        return _block(pos, vel, 24, ["v", "vv"])
    if name == "subwindow":  # window inside the periodic box: window clipping + images
        pos, vel = zeldovich(16, 2.0, 105)
        return _block(pos, vel, (20, 16, 24), ["x", "v", "xx", "vv"], bounds=((10.0, -5.0, 20.0), (60.0, 40.0, 95.0)))
    if name == "lattice":  # undisplaced lattice: every tet vertex on a grid plane
        return _block(lattice(16), np.zeros((16, 16, 16, 3)), 32, ["x"])
    if name == "refine":  # trilinear refinement, 2 levels
        pos, vel = zeldovich(8, 2.0, 106)
        return _block(pos, vel, 16, ["v"], reftol=0.2, maxlvl=2)
    if name == "nonperiodic":  # block mesh without a periodic box
        pos, vel = zeldovich(12, 0.5, 107)
        mass = np.random.default_rng(7).uniform(0.5, 2.0, (11, 11, 11))
        return _block(pos, vel, 20, ["x", "v", "vv"], mass=mass, periodic=False)
    if name == "tets":  # 'array' loader, simplex elements, random masses
        rng = np.random.default_rng(108)
        nt = 400
        c = rng.uniform(0.1, 0.9, (nt, 1, 3))
        pos = np.clip(c + rng.normal(0.0, 0.06, (nt, 4, 3)), 0.001, 0.999).reshape(-1, 3)
        vel = rng.normal(0.0, 1.0, pos.shape)
        conn = np.arange(4 * nt, dtype=np.int32).reshape(nt, 4)
        mass = rng.uniform(0.5, 1.5, nt)
        return dict(kind="array", pos=pos, vel=vel, mass=mass, conn=conn, periodic_box=None, n=(24, 24, 24),
                    bounds=((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)), fields=ALL, reftol=1.0, maxlvl=0)
    if name == "big_tet":  # one tet spanning a 64^3 grid: a bisection tree deeper than the main kernel's
        rng = np.random.default_rng(109)
        pos = 0.5 + (rng.random((4, 3)) - 0.5) * 0.9
        pos = pos[[0, 1, 2, 3]]
        return dict(kind="array", pos=pos, vel=rng.normal(size=(4, 3)), mass=None,
                    conn=np.arange(4, dtype=np.int32).reshape(1, 4), periodic_box=None, n=(64, 64, 64),
                    bounds=((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)), fields=["x", "v"], reftol=1.0, maxlvl=0)
    if name == "stretch":  # the stretch refinement criterion (not in the reference), 2 levels, threshold 2
        pos, vel = zeldovich(12, 3.0, 110)
        c = _block(pos, vel, 24, ["v"], reftol=2.0, maxlvl=2)
        c.update(refine_mode=1, refine_cell=(100.0 / 12,) * 3)
        return c
    raise KeyError(name)


NAMES = ["c1_small", "c2_small", "c2_order1", "rms3_vvonly", "subwindow", "lattice", "refine", "nonperiodic", "tets",
         "big_tet"]


def conn_of(c):
    import oracle as O

    if c["kind"] == "array":
        return c["conn"]
    return O.block_connectivity(c["pos"].shape[:3], c["periodic_box"] is not None)


def run_oracle(O, c, kind="restatement", counters=False):
    mass = None if c["mass"] is None else np.asarray(c["mass"]).reshape(-1)
    return O.voxelize(kind, n=c["n"], bounds=c["bounds"], pos=c["pos"].reshape(-1, 3), vel=c["vel"].reshape(-1, 3),
                      conn=conn_of(c), mass=mass, periodic_box=c["periodic_box"], fields=c["fields"],
                      reftol=c["reftol"], maxlvl=c["maxlvl"], counters=counters,
                      refine_mode=c.get("refine_mode", 0), refine_cell=c.get("refine_cell"))


def run_psi(PSI, c, grid=None, **kw):
    """Through the drop-in module, as a user of the reference would call it."""
    if grid is None:
        grid = PSI.Grid(type="cart", n=c["n"], bounds=c["bounds"], fields=c["fields"])
    mk = dict(loader=c["kind"], pos=c["pos"], vel=c["vel"])
    if c["mass"] is not None:
        mk["mass"] = c["mass"]
    if c["kind"] == "array":
        mk["connectivity"] = c["conn"]
    if c["periodic_box"] is not None:
        mk["periodic_box"] = c["periodic_box"]
    mesh = PSI.Mesh(**mk)
    if c.get("refine_mode"):
        kw.setdefault("refine_criterion", "stretch")
    PSI.voxels(grid=grid, mesh=mesh, refine_tolerance=c["reftol"], refine_max_lvl=c["maxlvl"], **kw)
    return {k: np.array(v) for k, v in grid.fields.items()}, grid, mesh


def total_mass(c):
    if c["mass"] is not None:
        return float(np.sum(c["mass"]))
    if c["kind"] == "array":
        return float(c["conn"].shape[0])
    s = c["pos"].shape[:3]
    return float(np.prod(s if c["periodic_box"] is not None else [v - 1 for v in s]))


def load_golden():
    """Cases stored by tests/golden/make_golden.py: {name: (case dict, expected fields)}."""
    import json
    import os

    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    out = {}
    for name, m in meta.items():
        c = dict(pos=z[f"{name}/in_pos"], vel=z[f"{name}/in_vel"], conn=z[f"{name}/in_conn"],
                 mass=z[f"{name}/in_mass"] if m["has_mass"] else None,
                 periodic_box=None if m["periodic_box"] is None else tuple(tuple(b) for b in m["periodic_box"]),
                 n=tuple(m["n"]), bounds=tuple(tuple(b) for b in m["bounds"]), fields=m["fields"],
                 reftol=m["reftol"], maxlvl=m["maxlvl"], kind="array")
        exp = {f.split("/out_")[1]: z[f] for f in z.files if f.startswith(f"{name}/out_")}
        out[name] = (c, exp)
    return out
