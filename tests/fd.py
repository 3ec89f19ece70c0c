"""Central finite differences of a density loss through the oracle.

The loss is L = sum_v (m_v / dV - rho_t,v)^2 over the voxels of a grid.  The
m field is linear in the tets, so moving one particle changes only the deposit
of the elements that contain it: with rho the full field and b(x) the deposit of
those elements alone,

    L(x +- h) = sum (rho_rest + b(x +- h)/dV - rho_t)^2,  rho_rest = rho - b(x)/dV,

and the central difference needs two oracle runs on a handful of elements.
This is how the reference's own C path (or its restatement) is differentiated
numerically, at any mesh size.
"""
from __future__ import annotations

import numpy as np


def block_elements_of(p: int, nside, periodic: bool) -> np.ndarray:
    """Elements of a block mesh that have particle p as a corner (src/PSI.c:636-656)."""
    nside = tuple(int(v) for v in nside)
    ne = nside if periodic else tuple(v - 1 for v in nside)
    ijk = np.unravel_index(int(p), nside)
    out = set()
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                e = [ijk[0] - a, ijk[1] - b, ijk[2] - c]
                if periodic:
                    e = [e[i] % ne[i] for i in range(3)]
                elif any(e[i] < 0 or e[i] >= ne[i] for i in range(3)):
                    continue
                out.add(int(np.ravel_multi_index(e, ne)))
    return np.array(sorted(out), dtype=np.int64)


def fd_loss_grad(O, kind, case, conn, rho, rho_t, p, ax, elems, h=1e-6):
    """dL/dpos[p, ax] by central differences of the oracle's deposit of `elems`.

    case: grid and mesh arrays as in tests/cases.py; conn: the full
    connectivity; rho: the m field of the whole mesh divided by dV."""
    n, bounds = case["n"], case["bounds"]
    dv = np.prod([(bounds[1][i] - bounds[0][i]) / n[i] for i in range(3)])
    pos = np.array(case["pos"], dtype=np.float64).reshape(-1, 3)
    sub = conn[elems]
    mass = None if case["mass"] is None else np.asarray(case["mass"]).reshape(-1)[elems]

    def dep(px):
        return O.voxelize(kind, n=n, bounds=bounds, pos=px, conn=sub, mass=mass,
                          periodic_box=case["periodic_box"], fields=[], reftol=case.get("reftol", 1.0),
                          maxlvl=case.get("maxlvl", 0))["m"] / dv

    b0 = dep(pos)
    pp, pm = pos.copy(), pos.copy()
    pp[p, ax] += h
    pm[p, ax] -= h
    bp, bm = dep(pp), dep(pm)
    a = rho - b0 - rho_t
    return float(np.sum((bp - bm) * (2.0 * a + bp + bm)) / (2.0 * h))
