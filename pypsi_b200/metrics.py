"""Per-voxel error of one set of grid fields against another.

Two measures per field, over voxels whose reference mass is positive:

* ``rel``  -- strict component-wise relative error |t - r| / |r| (components
  with r == 0 count as |t|).  Meaningful for ``m``; for vectors and tensors a
  component that is zero by cancellation makes it blow up in any
  implementation, so it is reported but not the acceptance bound.
* ``norm`` -- the error normalised by the voxel's own scale of that field:
  ``m``: m_ref; ``x``: max|x_ref|; ``v``: max(|v_ref|, sqrt(max diag vv_ref));
  ``xx``/``vv``: the largest diagonal entry of that voxel's tensor (which
  bounds every entry of a covariance); ``xv``: the larger of sqrt(max diag xx *
  max diag vv) and max|xv_ref| -- the reference's xv pairs its cross terms with
  the other variable (src/geometry.c:139-140), so it is not a covariance and the
  Cauchy-Schwarz scale alone does not bound it.  Each scale is floored at
  1e-12 of its mean over the grid.  This is the bound the parity tests enforce.
"""
from __future__ import annotations

import numpy as np


def _diagmax(t):
    return np.max(np.abs(np.diagonal(t, axis1=-2, axis2=-1)), axis=-1)


def _scales(ref: dict) -> dict:
    m = ref["m"]
    scales = {"m": np.abs(m)}
    if "x" in ref:
        scales["x"] = np.max(np.abs(ref["x"]), axis=-1)
    if "v" in ref:
        s = np.max(np.abs(ref["v"]), axis=-1)
        if "vv" in ref:
            s = np.maximum(s, np.sqrt(_diagmax(ref["vv"])))
        scales["v"] = s
    for f in ("xx", "vv"):
        if f in ref:
            scales[f] = _diagmax(ref[f])
    if "xv" in ref:
        s = np.max(np.abs(ref["xv"]).reshape(m.shape + (9,)), axis=-1)
        if "xx" in ref and "vv" in ref:
            s = np.maximum(s, np.sqrt(_diagmax(ref["xx"]) * _diagmax(ref["vv"])))
        scales["xv"] = s
    return scales


def error_maps(test: dict, ref: dict, scale_from: dict | None = None) -> dict:
    """Per-voxel normalised error of every field (the ``norm`` measure), as an
    array over the voxels where the scale source has positive mass.  The scales
    come from ``scale_from`` (default ``ref``), so maps of several pairs of
    results can be compared voxel by voxel."""
    sref = ref if scale_from is None else scale_from
    live = sref["m"] > 0
    nv = int(live.sum())
    scales = _scales(sref)
    out = {}
    for f, r in ref.items():
        if f not in test:
            continue
        dl = np.abs(test[f] - r)[live].reshape(nv, -1)
        sc = scales[f][live]
        floor = 1e-12 * float(np.mean(sc)) if sc.size else 0.0
        sc = np.maximum(sc, floor)
        out[f] = dl.max(axis=1) / np.where(sc > 0, sc, 1.0) if nv else np.zeros(0)
    return out


def field_errors(test: dict, ref: dict) -> dict:
    out = {}
    m = ref["m"]
    live = m > 0
    nv = int(live.sum())
    norms = error_maps(test, ref)
    for f, r in ref.items():
        t = test[f]
        d = np.abs(t - r)
        if nv == 0:
            out[f] = {"rel": 0.0, "norm": 0.0, "abs": float(d.max()) if d.size else 0.0}
            continue
        dl = d[live].reshape(nv, -1)
        rl = np.abs(r[live]).reshape(nv, -1)
        with np.errstate(divide="ignore", invalid="ignore"):
            rel = np.where(rl > 0, dl / rl, dl)
        out[f] = {"rel": float(rel.max()), "norm": float(norms[f].max()), "abs": float(d.max())}
    # voxels without reference mass must stay untouched up to rounding
    dead = ~live
    out["dead_m"] = float(np.abs(test["m"][dead]).max()) if dead.any() else 0.0
    return out


def mass_error(grid_m: np.ndarray, total_mass: float) -> float:
    """|1 - sum(m) / M_total|, the reference tutorial's global check."""
    return abs(1.0 - float(np.sum(grid_m)) / float(total_mass))
