"""Central finite differences of a loss on every grid field through the oracle.

The fields (m, x, v, xx, xv, vv) of a deposit into a zeroed grid are functions
of per-voxel sums that add over elements.  About fixed reference points r
(position) and s (velocity) of each voxel they are

    R0 = M,  Rx = M (X - r),  Rv = M (V - s),
    Rxx = M (XX + (X - r)(X - r)^T),  Rxv = M (XV + (X - r)(V - s)^T),  Rvv alike,

which the reference's online update (src/geometry.c:164-186) keeps exactly
(to rounding) whatever the order of the fragments.  Moving one particle
changes only the deposit of the elements that contain it, so with the full
deposit's sums R and the sums b(x) of those elements alone,

    L(x +- h) = L(fields(R - b(x) + b(x +- h))),

and the central difference needs two oracle runs on a handful of elements.
Taking r, s as the full deposit's means keeps the sums small, so nothing
cancels when the fields are rebuilt.
"""
from __future__ import annotations

import numpy as np

SECOND = {"xx": ("x", "x"), "xv": ("x", "v"), "vv": ("v", "v")}


def raw_sums(F: dict, r: np.ndarray, s: np.ndarray) -> dict:
    """Per-voxel sums of fields F about reference points r, s."""
    M = F["m"]
    out = {"m": M.copy()}
    d = {}
    if "x" in F:
        d["x"] = F["x"] - r
        out["x"] = M[..., None] * d["x"]
    if "v" in F:
        d["v"] = F["v"] - s
        out["v"] = M[..., None] * d["v"]
    for f, (a, b) in SECOND.items():
        if f in F:
            out[f] = M[..., None, None] * (F[f] + d[a][..., :, None] * d[b][..., None, :])
    return out


def fields_of(R: dict, r: np.ndarray, s: np.ndarray) -> dict:
    """The fields of per-voxel sums R about r, s (zero where R0 == 0)."""
    M = R["m"]
    live = M > 0
    safe = np.where(live, M, 1.0)
    out = {"m": M}
    mean = {}
    if "x" in R:
        mean["x"] = R["x"] / safe[..., None]
        out["x"] = np.where(live[..., None], r + mean["x"], 0.0)
    if "v" in R:
        mean["v"] = R["v"] / safe[..., None]
        out["v"] = np.where(live[..., None], s + mean["v"], 0.0)
    for f, (a, b) in SECOND.items():
        if f in R:
            cov = R[f] / safe[..., None, None] - mean[a][..., :, None] * mean[b][..., None, :]
            out[f] = np.where(live[..., None, None], cov, 0.0)
    return out


def loss(F: dict, W: dict) -> float:
    return float(sum(np.sum(W[f] * F[f]) for f in W))


def fd_grad(O, kind, case, conn, full: dict, W: dict, p: int, ax: int, elems, what="pos", h=1e-6) -> float:
    """dL/d(what[p, ax]) by central differences of the oracle's deposit of `elems`,
    L = sum over fields f of <W[f], field f>; `full` is the whole mesh's deposit."""
    names = list(full)
    flds = [f for f in names if f != "m"]
    pos = np.array(case["pos"], dtype=np.float64).reshape(-1, 3)
    vel = np.array(case["vel"], dtype=np.float64).reshape(-1, 3)
    sub = conn[elems]
    mass = None if case["mass"] is None else np.asarray(case["mass"]).reshape(-1)[elems]
    r = full["x"] if "x" in full else np.zeros(full["m"].shape + (3,))
    s = full["v"] if "v" in full else np.zeros(full["m"].shape + (3,))

    def dep(px, vx):
        return O.voxelize(kind, n=case["n"], bounds=case["bounds"], pos=px, vel=vx, conn=sub, mass=mass,
                          periodic_box=case["periodic_box"], fields=flds, reftol=case.get("reftol", 1.0),
                          maxlvl=case.get("maxlvl", 0))

    R = raw_sums(full, r, s)
    b0 = raw_sums(dep(pos, vel), r, s)
    rest = {f: R[f] - b0[f] for f in R}
    vals = []
    for sign in (1.0, -1.0):
        px, vx = pos.copy(), vel.copy()
        (px if what == "pos" else vx)[p, ax] += sign * h
        b = raw_sums(dep(px, vx), r, s)
        vals.append(loss(fields_of({f: rest[f] + b[f] for f in R}, r, s), W))
    return (vals[0] - vals[1]) / (2.0 * h)
