"""The finite-difference checker of the adjoint tests, on the CPU.

Moving one particle and re-depositing only the elements that contain it must
give the same central difference as re-depositing the whole mesh (the deposit
is linear in the tets), for the reference's C path and for its restatement.
"""
import numpy as np
import pytest

import cases
from fd import block_elements_of, fd_loss_grad


def test_block_elements_of_periodic_and_open():
    assert len(block_elements_of(0, (4, 4, 4), True)) == 8
    assert list(block_elements_of(0, (4, 4, 4), False)) == [0]
    # the particle at the far corner of an open block belongs to the last element only
    assert list(block_elements_of(63, (4, 4, 4), False)) == [26]


@pytest.mark.parametrize("kind", ["restatement", "reference"])
def test_subset_fd_equals_whole_mesh_fd(oracle, kind):
    if not oracle.available(kind):
        pytest.skip(f"{kind} library not built")
    from pypsi_b200.synth import zeldovich

    pos, vel = zeldovich(6, 1.0, 77)
    case = cases._block(pos, vel, 12, [])
    conn = cases.conn_of(case)
    n, bounds = case["n"], case["bounds"]
    dv = np.prod([(bounds[1][i] - bounds[0][i]) / n[i] for i in range(3)])
    rng = np.random.default_rng(1)
    flat = pos.reshape(-1, 3)
    rho_t = oracle.voxelize(kind, n=n, bounds=bounds, pos=flat + rng.normal(0, 0.4, flat.shape), conn=conn,
                            periodic_box=case["periodic_box"])["m"] / dv

    def loss(px):
        rho = oracle.voxelize(kind, n=n, bounds=bounds, pos=px, conn=conn, periodic_box=case["periodic_box"])["m"] / dv
        return float(np.sum((rho - rho_t) ** 2)), rho

    l0, rho = loss(flat)
    h = 1e-5
    for p, ax in [(0, 0), (37, 1), (100, 2), (215, 0)]:
        sub = fd_loss_grad(oracle, kind, case, conn, rho, rho_t, p, ax, block_elements_of(p, (6, 6, 6), True), h=h)
        pp, pm = flat.copy(), flat.copy()
        pp[p, ax] += h
        pm[p, ax] -= h
        whole = (loss(pp)[0] - loss(pm)[0]) / (2 * h)
        assert abs(sub - whole) <= 1e-6 * max(abs(whole), 1e-3), (p, ax, sub, whole)


@pytest.mark.parametrize("refine", [(1.0, 0), (0.2, 2)])
@pytest.mark.parametrize("kind", ["restatement", "reference"])
def test_subset_fd_of_every_field_equals_whole_mesh_fd(oracle, kind, refine):
    """The finite differences of a loss on every field (tests/fd_fields.py):
    re-depositing the elements around one particle, through per-voxel sums,
    gives the same central difference as re-depositing the whole mesh, for
    positions and velocities, with and without refinement of the elements."""
    if not oracle.available(kind):
        pytest.skip(f"{kind} library not built")
    from fd_fields import fd_grad, loss
    from pypsi_b200.synth import zeldovich

    pos, vel = zeldovich(6, 1.0, 78)
    fields = ["x", "v", "xx", "xv", "vv"]
    case = cases._block(pos, vel, 12, fields, reftol=refine[0], maxlvl=refine[1])
    conn = cases.conn_of(case)
    flat, vflat = pos.reshape(-1, 3), vel.reshape(-1, 3)

    def dep(px, vx, k=kind, counters=False):
        return oracle.voxelize(k, n=case["n"], bounds=case["bounds"], pos=px, vel=vx, conn=conn,
                               periodic_box=case["periodic_box"], fields=fields, reftol=refine[0],
                               maxlvl=refine[1], counters=counters)

    if refine[1]:  # the tolerance refines some elements (the restatement counts the tets)
        assert dep(flat, vflat, "restatement", True)[1]["tets"] > 6 * 6 ** 3

    full = dep(flat, vflat)
    rng = np.random.default_rng(2)
    live = full["m"] > 0
    h = 1e-5
    for f in ["m"] + fields:
        W = {f: rng.normal(size=full[f].shape) * live.reshape(live.shape + (1,) * (full[f].ndim - 3))}
        for what, p, ax in [("pos", 5, 0), ("pos", 101, 2), ("vel", 37, 1), ("vel", 200, 0)]:
            if f in ("m", "x", "xx") and what == "vel":
                continue
            sub = fd_grad(oracle, kind, case, conn, full, W, p, ax, block_elements_of(p, (6, 6, 6), True), what, h)
            a, b = flat.copy(), vflat.copy()
            (a if what == "pos" else b)[p, ax] += h
            lp = loss(dep(a, b), W)
            a, b = flat.copy(), vflat.copy()
            (a if what == "pos" else b)[p, ax] -= h
            lm = loss(dep(a, b), W)
            whole = (lp - lm) / (2 * h)
            assert abs(sub - whole) <= 1e-5 * max(abs(whole), 1e-3), (f, what, p, ax, sub, whole)
