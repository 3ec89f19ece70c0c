"""The oracle's element queries and phase-space samples pinned to the
reference's own (psi_rtree_* of src/rtree.c and psi_sample_vdf of
src/cpsi.c:177-275, compiled in oracle/_ref): the same elements in the same
order and the same samples bit for bit while the reference's tree is one leaf
(at most 32 elements), the same sets beyond."""
import numpy as np
import pytest

import oracle as O
from vdf_cases import LARGE, SMALL, make, sorted_samples, vdf


def need_reference(oracle):
    if not oracle.available("reference"):
        pytest.skip("the reference is not compiled here")


@pytest.mark.parametrize("name", SMALL + LARGE)
def test_query_matches_reference(oracle, name):
    need_reference(oracle)
    c = make(name)
    win = O.tree_window(c["periodic_box"])
    rng = np.random.default_rng(5)
    for _ in range(8):
        lo = rng.uniform(-0.1, 0.9, 3)
        box = (tuple(lo), tuple(lo + rng.uniform(0.0, 0.4, 3)))
        ref = O.query_elements("reference", c["pos"], c["conn"], win, box, c["periodic_box"])
        got = O.query_elements("restatement", c["pos"], c["conn"], win, box, c["periodic_box"])
        if name in SMALL:
            assert np.array_equal(got, ref), (name, box)
        else:
            assert np.array_equal(np.sort(got), np.sort(ref)), (name, box)


@pytest.mark.parametrize("tree", [False, True])
@pytest.mark.parametrize("name", SMALL + LARGE)
def test_vdf_matches_reference(oracle, name, tree):
    need_reference(oracle)
    c = make(name)
    nonempty = 0
    for p in c["points"]:
        r_rho, r_vel = vdf(c, "reference", p, tree)
        g_rho, g_vel = vdf(c, "restatement", p, tree)
        nonempty += len(r_rho) > 0
        if name in SMALL:
            assert np.array_equal(g_rho, r_rho) and np.array_equal(g_vel, r_vel), (name, p)
        else:
            assert np.array_equal(sorted_samples(g_rho, g_vel), sorted_samples(r_rho, r_vel)), (name, p)
    if tree or c["periodic_box"] is not None:
        assert nonempty > 0


def test_vdf_without_tree_on_an_open_mesh_sees_only_the_origin(oracle):
    """The tree PSI.VDF builds for itself culls against mesh.box, which is zero
    for an open mesh: only elements whose box holds the origin survive."""
    c = make("open4_mild")
    for p in c["points"][1:]:
        assert len(vdf(c, "restatement", p, tree=False)[0]) == 0
    hit = [len(vdf(c, "restatement", p, tree=True)[0]) for p in c["points"][1:]]
    assert max(hit) >= 1


def test_vdf_single_stream_density(oracle):
    """An undisplaced lattice: every interior point lies in exactly one tet of one
    element (away from faces), whose density is the element mass / its volume."""
    q = (np.arange(4) + 0.5) / 4
    pos = np.stack(np.meshgrid(q, q, q, indexing="ij"), -1).reshape(-1, 3)
    conn = O.block_connectivity((4, 4, 4), False)
    vel = np.tile([1.0, -2.0, 0.5], (len(pos), 1))
    mass = np.full(conn.shape[0], 6.0)
    cell = 1.0 / 4
    for p in ([0.3, 0.41, 0.52], [0.61, 0.27, 0.33]):
        rho, v = O.sample_vdf("restatement", pos, conn, p, vel=vel, mass=mass, window=O.tree_window(None))
        assert len(rho) == 1
        assert abs(rho[0] - 1.0 / (cell ** 3 / 6)) <= 1e-9 * rho[0]
        assert np.allclose(v[0], [1.0, -2.0, 0.5], rtol=0, atol=1e-12)


def test_vdf_on_faces_edges_and_vertices_matches_reference(oracle):
    """Points on the shared faces, edges and vertices of an undisplaced lattice:
    every tet whose barycentric coordinates there are all >= 0 gives a sample,
    so a point on a face or a vertex is counted by several tets -- the count
    and the values equal the reference's."""
    need_reference(oracle)
    q = (np.arange(4) + 0.5) / 4
    pos = np.stack(np.meshgrid(q, q, q, indexing="ij"), -1).reshape(-1, 3)
    conn = O.block_connectivity((4, 4, 4), False)
    vel = np.random.default_rng(2).normal(size=pos.shape)
    mass = np.random.default_rng(3).uniform(0.5, 1.5, conn.shape[0])
    h = 0.25
    pts = [pos[21], pos[22] + [0, 0, h / 2], pos[21] + [h / 2, h / 2, 0], pos[21] + [h / 2, h / 2, h / 2],
           pos[42] + [h / 3, h / 3, h / 3], pos[5] + [0, h / 4, h / 2]]
    multi = 0
    for p in pts:
        kw = dict(vel=vel, mass=mass, window=O.tree_window(None))
        r = O.sample_vdf("reference", pos, conn, p, **kw)
        g = O.sample_vdf("restatement", pos, conn, p, **kw)
        assert np.array_equal(g[0], r[0]) and np.array_equal(g[1], r[1]), p
        multi += len(r[0]) > 1
    assert multi > 0  # some points sit on shared faces
