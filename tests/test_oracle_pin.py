"""Pins the CPU oracle before it is trusted as the checker.

* the C restatement (oracle/psi_oracle.c) equals the reference's own sources
  compiled unchanged (oracle/_ref) bit for bit on every parity case;
* both equal the committed golden fixtures made from the reference;
* known answers: a tet inside one voxel, the undisplaced lattice, mass
  conservation (the tutorial's only published check, Tutorial.ipynb:67-75,186,414).
"""
import numpy as np
import pytest

from cases import NAMES, load_golden, make, run_oracle, total_mass
from pypsi_b200.metrics import mass_error

CPU_NAMES = [n for n in NAMES if n != "c2_small"] + ["c2_small"]


@pytest.mark.parametrize("name", CPU_NAMES)
def test_restatement_equals_reference_bitwise(oracle, name):
    if not oracle.available("reference"):
        pytest.skip("reference sources were not compiled on this machine (golden fixtures still pin the oracle)")
    c = make(name)
    a = run_oracle(oracle, c, "restatement")
    b = run_oracle(oracle, c, "reference")
    assert sorted(a) == sorted(b)
    for f in a:
        assert np.array_equal(a[f], b[f]), f"{name}: field {f} differs"


@pytest.mark.parametrize("gname", sorted(load_golden()))
def test_restatement_matches_golden(oracle, gname):
    c, exp = load_golden()[gname]
    out = run_oracle(oracle, c, "restatement")
    for f, e in exp.items():
        assert np.array_equal(out[f], e), f"{gname}: field {f}"


@pytest.mark.parametrize("gname", sorted(load_golden()))
def test_reference_matches_golden(oracle, gname):
    if not oracle.available("reference"):
        pytest.skip("reference library absent")
    c, exp = load_golden()[gname]
    out = run_oracle(oracle, c, "reference")
    for f, e in exp.items():
        assert np.array_equal(out[f], e), f"{gname}: field {f}"


def test_tet_inside_one_voxel(oracle):
    """m = mass, x = centroid, xx = the tet's covariance (1/20) sum (v_i - c)(v_i - c)^T."""
    rng = np.random.default_rng(3)
    v = np.array([0.31, 0.32, 0.33]) + rng.uniform(0.0, 0.05, (4, 3))
    c = dict(kind="array", pos=v, vel=np.zeros((4, 3)), mass=np.array([2.5]), conn=np.arange(4, dtype=np.int32)[None],
             periodic_box=None, n=(2, 2, 2), bounds=((0, 0, 0), (1, 1, 1)), fields=["x", "xx"], reftol=1.0, maxlvl=0)
    out = run_oracle(oracle, c)
    m = out["m"]
    assert m[0, 0, 0] == pytest.approx(2.5, rel=1e-14)
    assert np.count_nonzero(m) == 1
    cen = v.mean(axis=0)
    np.testing.assert_allclose(out["x"][0, 0, 0], cen, rtol=1e-14)
    cov = sum(np.outer(p - cen, p - cen) for p in v) / 20.0
    np.testing.assert_allclose(out["xx"][0, 0, 0], cov, rtol=1e-10, atol=1e-16)


def test_lattice_gives_mass_over_eight(oracle):
    """Undisplaced lattice on a grid of twice its resolution: each voxel is an
    eighth of exactly one element."""
    out = run_oracle(oracle, make("lattice"))
    np.testing.assert_allclose(out["m"], 0.125, rtol=0, atol=1e-15)


@pytest.mark.parametrize("name", ["c1_small", "c2_small", "rms3_vvonly", "lattice", "refine", "big_tet", "tets"])
def test_mass_conservation(oracle, name):
    c = make(name)
    out = run_oracle(oracle, c)
    assert mass_error(out["m"], total_mass(c)) < 1e-13


def test_counters(oracle):
    out, cnt = run_oracle(oracle, make("c1_small"), counters=True)
    assert cnt["errors"] == 0
    assert cnt["tets"] == 6 * 16 ** 3
    assert cnt["max_verts"] <= 32
    assert 10 < cnt["fragments"] / cnt["tets"] < 25


def test_exact_oracle_agrees_where_the_reference_is_well_conditioned(oracle):
    """The quad-precision oracle runs the same algorithm: on a case without tiny
    fragments it agrees with the FP64 restatement to FP64 rounding, and on
    random simplex tets it exposes the reference's own rounding in the second
    moments of sliver voxels (which the mixed-precision tests allow for)."""
    from pypsi_b200.metrics import field_errors

    c = make("c2_order1")
    r = run_oracle(oracle, c, "restatement")
    e = run_oracle(oracle, c, "exact")
    errs = field_errors(r, e)
    assert max(v["norm"] for k, v in errs.items() if k != "dead_m") <= 1e-12, errs
    c = make("tets")
    r = run_oracle(oracle, c, "restatement")
    e = run_oracle(oracle, c, "exact")
    errs = field_errors(r, e)
    assert errs["m"]["rel"] <= 1e-9, errs["m"]
    assert errs["xx"]["norm"] > 1e-6, errs["xx"]  # the reference's own error in sliver voxels
    assert abs(e["m"].sum() - c["mass"].sum()) <= 1e-12 * c["mass"].sum()


def test_stretch_criterion_limits_in_the_oracle(oracle):
    """The stretch refinement criterion (an extension the GPU library shares):
    a huge threshold refines nothing, a tiny one refines every element to the
    maximum level, and mass is conserved either way."""
    c = make("stretch")
    n = c["pos"].shape[0]
    for T, want in [(1.0e9, 6 * n ** 3), (1.0e-9, 6 * n ** 3 * 64)]:
        c["reftol"] = T
        out, cnt = run_oracle(oracle, c, counters=True)
        assert cnt["tets"] == want, (T, cnt["tets"])
        assert abs(out["m"].sum() / n ** 3 - 1.0) < 1e-13
    c["reftol"] = 2.0
    _, cnt = run_oracle(oracle, c, counters=True)
    assert 6 * n ** 3 < cnt["tets"] < 6 * n ** 3 * 64, cnt["tets"]
