"""Reader of tests/golden/golden_modes.npz (annihilation and phase-space
samples of the reference, written by tests/golden/make_golden_modes.py)."""
from __future__ import annotations

import json
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_modes.npz")


def load():
    z = np.load(PATH)
    meta = json.loads(bytes(z["meta"]).decode())
    return z, meta


def ann_case(z, meta, name):
    """The stored annihilation case as an ann_cases-style dict, and the reference's m."""
    c = dict(meta["ann"][name])
    c["n"] = tuple(c["n"])
    c["pos"] = z[f"ann/{name}/pos"]
    c["conn"] = z[f"ann/{name}/conn"]
    c["mass"] = z[f"ann/{name}/mass"] if c.pop("has_mass") else None
    return c, z[f"ann/{name}/m"]


def vdf_case(z, meta, name):
    """The stored sampling case as a vdf_cases-style dict, and per tree flag the
    reference's samples (offsets, rho, vel)."""
    c = dict(meta["vdf"][name])
    for k in ("pos", "conn", "vel", "mass", "points"):
        c[k] = z[f"vdf/{name}/{k}"]
    want = {t: (z[f"vdf/{name}/tree{t}/off"], z[f"vdf/{name}/tree{t}/rho"], z[f"vdf/{name}/tree{t}/vel"])
            for t in (0, 1)}
    return c, want
