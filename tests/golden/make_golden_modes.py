"""Generate tests/golden/golden_modes.npz from the reference implementation.

    python tests/golden/make_golden_modes.py

Runs PyPSI's own annihilation deposit (psi_voxels with PSI_MODE_ANNIHILATION)
and its phase-space sampling (psi_sample_vdf over its own R*-tree), both
compiled unchanged into oracle/_ref/libpsiref.so, on the small seeded cases of
tests/ann_cases.py and tests/vdf_cases.py whose reference tree is one leaf (so
the reference's order is the one this library reproduces), and stores inputs,
arguments and outputs.  They carry the reference's behaviour to machines where
its sources are absent.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import ann_cases  # noqa: E402
import oracle as O  # noqa: E402
import vdf_cases  # noqa: E402


def main():
    O.build()
    data, meta = {}, {"ann": {}, "vdf": {}}
    for name in ann_cases.SMALL + ["degenerate"]:
        c = ann_cases.make(name)
        out = ann_cases.run_oracle(c, "reference")["m"]
        data[f"ann/{name}/pos"] = c["pos"]
        data[f"ann/{name}/conn"] = c["conn"]
        if c["mass"] is not None:
            data[f"ann/{name}/mass"] = np.asarray(c["mass"])
        data[f"ann/{name}/m"] = out
        meta["ann"][name] = {k: c[k] for k in ("n", "bounds", "periodic_box", "reftol", "maxlvl")}
        meta["ann"][name]["has_mass"] = c["mass"] is not None
    for name in vdf_cases.SMALL:
        c = vdf_cases.make(name)
        for k in ("pos", "conn", "vel", "mass", "points"):
            data[f"vdf/{name}/{k}"] = c[k]
        for tree in (False, True):
            res = [vdf_cases.vdf(c, "reference", p, tree) for p in c["points"]]
            off = np.concatenate([[0], np.cumsum([len(r[0]) for r in res])]).astype(np.int64)
            data[f"vdf/{name}/tree{int(tree)}/off"] = off
            data[f"vdf/{name}/tree{int(tree)}/rho"] = np.concatenate([r[0] for r in res])
            data[f"vdf/{name}/tree{int(tree)}/vel"] = np.concatenate([r[1] for r in res]).reshape(-1, 3)
        meta["vdf"][name] = {k: c[k] for k in ("periodic_box", "reftol", "maxlvl")}
    data["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "golden_modes.npz"), **data)
    print("wrote", os.path.join(HERE, "golden_modes.npz"), sorted(meta["ann"]), sorted(meta["vdf"]))


if __name__ == "__main__":
    main()
