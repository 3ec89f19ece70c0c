"""Annihilation and PSI.VDF on the GPU against the reference's own outputs
stored in tests/golden/golden_modes.npz, bit for bit: the same check as the
live comparisons with the compiled reference, on machines without it."""
import numpy as np
import pytest

import golden_modes as G

pytestmark = pytest.mark.gpu

Z, META = G.load()


def _tuples(b):
    return None if b is None else tuple(tuple(float(v) for v in r) for r in b)


@pytest.mark.parametrize("name", sorted(META["ann"]))
def test_annihilation_matches_golden(gpu, name):
    from test_gpu_annihilation import run_gpu

    c, want = G.ann_case(Z, META, name)
    c["bounds"] = _tuples(c["bounds"])
    c["periodic_box"] = _tuples(c["periodic_box"])
    got, _ = run_gpu(gpu, c)
    assert np.array_equal(got, want, equal_nan=True), name


@pytest.mark.parametrize("name", sorted(META["vdf"]))
def test_vdf_matches_golden(gpu, name):
    from test_gpu_vdf import module_mesh

    c, want = G.vdf_case(Z, META, name)
    c["periodic_box"] = _tuples(c["periodic_box"])
    mesh = module_mesh(gpu, c)
    tree = gpu.RStarTree(mesh)
    for t in (0, 1):
        off, rho, vel = want[t]
        for i, p in enumerate(c["points"]):
            kw = dict(refine_tolerance=c["reftol"], refine_max_lvl=c["maxlvl"])
            r, v = gpu.VDF(mesh, tuple(p), tree, **kw) if t else gpu.VDF(mesh, tuple(p), **kw)
            assert np.array_equal(r, rho[off[i]:off[i + 1]]) and np.array_equal(v, vel[off[i]:off[i + 1]]), (
                name, t, i)
