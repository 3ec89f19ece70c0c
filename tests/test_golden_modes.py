"""The oracle's annihilation and phase-space samples against the reference's
own outputs stored in tests/golden/golden_modes.npz: bit for bit, without the
reference's sources (the fixtures are regenerated by
tests/golden/make_golden_modes.py where they are present)."""
import numpy as np
import pytest

import ann_cases
import golden_modes as G
import vdf_cases

Z, META = G.load()


@pytest.mark.parametrize("name", sorted(META["ann"]))
def test_annihilation_oracle_matches_golden(oracle, name):
    c, want = G.ann_case(Z, META, name)
    got = ann_cases.run_oracle(c)["m"]
    assert np.array_equal(got, want, equal_nan=True), name


@pytest.mark.parametrize("name", sorted(META["vdf"]))
def test_vdf_oracle_matches_golden(oracle, name):
    c, want = G.vdf_case(Z, META, name)
    for tree in (0, 1):
        off, rho, vel = want[tree]
        for i, p in enumerate(c["points"]):
            r, v = vdf_cases.vdf(c, "restatement", p, bool(tree))
            assert np.array_equal(r, rho[off[i]:off[i + 1]]) and np.array_equal(v, vel[off[i]:off[i + 1]]), (
                name, tree, i)


def test_goldens_regenerate_identically(oracle):
    """Where the reference is compiled, the stored cases are still what the case
    builders make (so the fixtures and the live tests check the same inputs)."""
    for name in META["ann"]:
        c, _ = G.ann_case(Z, META, name)
        assert np.array_equal(c["pos"], ann_cases.make(name)["pos"]), name
    for name in META["vdf"]:
        c, _ = G.vdf_case(Z, META, name)
        assert np.array_equal(c["pos"], vdf_cases.make(name)["pos"]), name
