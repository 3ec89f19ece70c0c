"""The oracle's annihilation mode pinned to the reference's own (src/cpsi.c:115-158,
compiled in oracle/_ref): bit for bit wherever the reference's R*-tree is a
single leaf (at most 32 kept elements), to the rounding of a reordered sum
beyond, and to the quad-precision oracle within the reference's own error."""
import numpy as np
import pytest

from ann_cases import LARGE, SMALL, make, run_oracle


def need_reference(oracle):
    if not oracle.available("reference"):
        pytest.skip("the reference is not compiled here")


@pytest.mark.parametrize("name", SMALL)
def test_restatement_equals_reference_bitwise(oracle, name):
    need_reference(oracle)
    c = make(name)
    ref = run_oracle(c, "reference")["m"]
    out, cnt = run_oracle(c, counters=True)
    assert np.array_equal(out["m"], ref), name
    assert cnt["errors"] == 0 and cnt["fragments"] > 0 and cnt["elements_kept"] <= 32


def test_degenerate_tet_as_the_reference(oracle):
    """A tet with a repeated vertex has zero volume: the reference's density
    mass / volume is infinite and the voxels it touches get inf or NaN."""
    need_reference(oracle)
    c = make("degenerate")
    ref = run_oracle(c, "reference")["m"]
    out = run_oracle(c)["m"]
    assert not np.isfinite(ref).all()
    assert np.array_equal(out, ref, equal_nan=True)


@pytest.mark.parametrize("name", LARGE)
def test_restatement_near_reference(oracle, name):
    """More than 32 elements: the reference's tree visits partners in another
    order, so the per-voxel sums agree to rounding."""
    need_reference(oracle)
    c = make(name)
    ref = run_oracle(c, "reference")["m"]
    out, cnt = run_oracle(c, counters=True)
    assert cnt["elements_kept"] > 32
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.abs(out["m"] - ref).max() <= 1e-14 * scale


@pytest.mark.parametrize("name", ["block3", "periodic3"])
def test_exact_oracle(oracle, name):
    c = make(name)
    ex = run_oracle(c, "exact")["m"]
    out = run_oracle(c)["m"]
    assert np.abs(out - ex).max() <= 1e-10 * np.abs(ex).max()


def test_two_identical_tets(oracle):
    """One tet of mass M and volume V against itself: each voxel gets
    rho^2 x (its share of the volume), summing to M^2 / V; with two elements of
    the same tet, four pairs give 4 M^2 / V."""
    p = np.array([[0.1, 0.1, 0.1], [0.9, 0.2, 0.15], [0.2, 0.85, 0.1], [0.15, 0.2, 0.9]])
    vol = abs(np.linalg.det(p[1:] - p[0])) / 6
    for k in (1, 2):
        conn = np.tile(np.arange(4, dtype=np.int32), (k, 1))
        out = oracle.voxelize("restatement", (6, 6, 6), ((0, 0, 0), (1, 1, 1)), p, conn, mass=np.full(k, 2.0),
                              mode="annihilation")["m"]
        assert abs(out.sum() - k * k * 4.0 / vol) <= 1e-12 * k * k * 4.0 / vol


def test_disjoint_tets_deposit_nothing(oracle):
    p = np.array([[0.1, 0.1, 0.1], [0.3, 0.1, 0.1], [0.1, 0.3, 0.1], [0.1, 0.1, 0.3],
                  [0.6, 0.6, 0.6], [0.9, 0.6, 0.6], [0.6, 0.9, 0.6], [0.6, 0.6, 0.9]])
    conn = np.array([[0, 1, 2, 3], [4, 5, 6, 7]], dtype=np.int32)
    out, cnt = oracle.voxelize("restatement", (5, 5, 5), ((0, 0, 0), (1, 1, 1)), p, conn, mode="annihilation",
                               counters=True)
    # only the two self pairs
    assert cnt["tet_images"] == 2
    vol0 = abs(np.linalg.det(p[1:4] - p[0])) / 6
    vol1 = abs(np.linalg.det(p[5:8] - p[4])) / 6
    assert abs(out["m"].sum() - (1 / vol0 + 1 / vol1)) <= 1e-12 * (1 / vol0 + 1 / vol1)
