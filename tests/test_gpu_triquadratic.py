"""Triquadratic (27-node) elements, the first "next" row of the path.

A mesh of 27-node cubes (node (a,b,c) of element (i,j,k) is lattice point
(2i+a, 2j+b, 2k+c), node order 9a+3b+c) with a smooth displacement, clipped by a
window, deposited through the drop-in module and compared with the reference's
own C code (src/refine.c:152-221 refines such elements through the triquadratic
interpolation of src/refine.c:321-345): FP64 bit for bit at refinement levels
0 and 2, mixed within 1e-5 of the FP64-central result and of the reference.
"""
import numpy as np
import pytest

from cases import run_oracle, run_psi
from pypsi_b200.metrics import error_maps, field_errors

pytestmark = pytest.mark.gpu

ALL = ["x", "v", "xx", "xv", "vv"]


def _quad_case(ne=6, maxlvl=0, reftol=1.0, seed=3):
    rng = np.random.default_rng(seed)
    nn = 2 * ne + 1
    g = np.stack(np.meshgrid(*([np.arange(nn) / (nn - 1)] * 3), indexing="ij"), axis=-1)
    ph = rng.uniform(0, 2 * np.pi, 3)
    pos = g.copy()
    for a in range(3):
        pos[..., a] += 0.03 * np.sin(2 * np.pi * g[..., (a + 1) % 3] + ph[a]) + 0.02 * np.sin(4 * np.pi * g[..., a])
    vel = rng.normal(0, 1, pos.shape)
    conn = np.empty((ne, ne, ne, 27), dtype=np.int32)
    i, j, k = np.meshgrid(np.arange(ne), np.arange(ne), np.arange(ne), indexing="ij")
    for a in range(3):
        for b in range(3):
            for c in range(3):
                conn[..., 9 * a + 3 * b + c] = ((2 * i + a) * nn + (2 * j + b)) * nn + (2 * k + c)
    return dict(kind="array", pos=pos.reshape(-1, 3), vel=vel.reshape(-1, 3), mass=rng.uniform(0.5, 1.5, ne ** 3),
                conn=conn.reshape(-1, 27), periodic_box=None, n=(20, 20, 20),
                bounds=((0.05, 0.05, 0.05), (0.95, 0.95, 0.95)), fields=ALL, reftol=reftol, maxlvl=maxlvl)


@pytest.mark.parametrize("maxlvl,reftol", [(0, 1.0), (2, 0.02)])
def test_triquadratic_fp64_bitwise_against_reference(gpu, oracle, maxlvl, reftol):
    # the compiled reference where it travelled with the tree, else the restatement pinned to it
    kind = "reference" if oracle.available("reference") else "restatement"
    c = _quad_case(maxlvl=maxlvl, reftol=reftol)
    ref, _ = run_oracle(oracle, c, kind=kind, counters=True)
    out, _, _ = run_psi(gpu, c, precision="fp64")
    st = gpu.last_stats()
    if maxlvl:
        assert st["tets"] > 6 * 6 ** 3  # the tolerance refined some elements
    else:
        assert st["tets"] == 6 * 6 ** 3
    for f in ref:
        assert np.array_equal(out[f], ref[f]), (f, np.abs(out[f] - ref[f]).max())


def test_triquadratic_mixed(gpu, oracle):
    kind = "reference" if oracle.available("reference") else "restatement"
    c = _quad_case(maxlvl=2, reftol=0.02)
    ref = run_oracle(oracle, c, kind=kind)
    central, _, _ = run_psi(gpu, c, precision="fp64-central")
    mixed, _, _ = run_psi(gpu, c, precision="mixed")
    errs = field_errors(mixed, central)
    assert errs["m"]["rel"] <= 1e-5 and max(e["norm"] for f, e in errs.items() if f != "dead_m") <= 1e-5, errs
    e_mr = error_maps(mixed, ref, scale_from=central)
    e_rc = error_maps(ref, central)
    for f in e_mr:
        assert (e_mr[f] <= 1e-5 + e_rc[f]).all(), f
