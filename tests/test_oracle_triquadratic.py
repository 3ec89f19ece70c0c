"""The oracle's triquadratic (27-node) elements pinned to the reference's own
(src/refine.c:152-221, :321-345, compiled in oracle/_ref): density fields of
every order, annihilation and phase-space samples, bit for bit, at refinement
levels 0 to 2."""
import numpy as np
import pytest

import oracle as O


def quad_case(ne=3, seed=3):
    from test_gpu_triquadratic import _quad_case

    return _quad_case(ne=ne, seed=seed)


def need_reference(oracle):
    if not oracle.available("reference"):
        pytest.skip("the reference is not compiled here")


@pytest.mark.parametrize("maxlvl,reftol", [(0, 1.0), (1, 0.05), (2, 0.02)])
def test_density_matches_reference(oracle, maxlvl, reftol):
    need_reference(oracle)
    q = quad_case()
    kw = dict(n=(12, 12, 12), bounds=q["bounds"], pos=q["pos"], conn=q["conn"], vel=q["vel"], mass=q["mass"],
              fields=("x", "v", "xx", "xv", "vv"), reftol=reftol, maxlvl=maxlvl)
    ref = O.voxelize("reference", **kw)
    got, cnt = O.voxelize("restatement", counters=True, **kw)
    for f in ref:
        assert np.array_equal(got[f], ref[f]), (maxlvl, f)
    assert cnt["tets"] >= 6 * 27 and cnt["errors"] == 0
    if maxlvl:
        assert cnt["tets"] > 6 * 27  # the tolerance refined some elements


@pytest.mark.parametrize("maxlvl,reftol", [(0, 1.0), (1, 0.05)])
def test_annihilation_matches_reference(oracle, maxlvl, reftol):
    need_reference(oracle)
    q = quad_case()
    kw = dict(n=(10, 10, 10), bounds=q["bounds"], pos=q["pos"], conn=q["conn"], mass=q["mass"], reftol=reftol,
              maxlvl=maxlvl, mode="annihilation")
    ref = O.voxelize("reference", **kw)["m"]
    got = O.voxelize("restatement", **kw)["m"]
    assert np.abs(ref).max() > 0 and np.array_equal(got, ref)


def test_vdf_matches_reference(oracle):
    need_reference(oracle)
    q = quad_case()
    n = 0
    for p in np.random.default_rng(4).uniform(0.1, 0.9, (12, 3)):
        kw = dict(vel=q["vel"], mass=q["mass"], window=O.tree_window(None), reftol=0.01, maxlvl=1)
        r = O.sample_vdf("reference", q["pos"], q["conn"], p, **kw)
        g = O.sample_vdf("restatement", q["pos"], q["conn"], p, **kw)
        assert np.array_equal(g[0], r[0]) and np.array_equal(g[1], r[1])
        n += len(r[0])
    assert n > 0
