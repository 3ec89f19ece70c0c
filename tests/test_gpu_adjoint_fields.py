"""Adjoint of every field (psib_voxels_adjoint_fields via deposit_fields).

For a loss L = sum over voxels of <W, field> on one field at a time -- m, x,
v, xx, xv, vv with random weights W -- the gradient with respect to particle
positions and velocities from the adjoint kernel is checked against central
finite differences (h = 1e-6) of the reference's own C path (oracle/_ref; the
pinned restatement where it is absent), moving one particle (or its velocity)
and re-depositing the elements that contain it through per-voxel sums
(tests/fd_fields.py).  Element-mass gradients are checked against the deposit
of each element alone scaled (every field's sums are linear in a tet's mass).
Refined elements (8-node trilinear and 27-node triquadratic, midpoint criterion)
are checked the same way, the finite differences refining as the reference does.
"""
import numpy as np
import pytest

import cases
from fd import block_elements_of
from fd_fields import fd_grad, fields_of, loss, raw_sums

pytestmark = pytest.mark.gpu

ALL = ["x", "v", "xx", "xv", "vv"]
RTOL = 1e-6   # |adjoint - finite difference| <= RTOL * max |gradient| of that loss


def _kind(O):
    return "reference" if O.available("reference") else "restatement"


def _weights(F, f, seed):
    rng = np.random.default_rng(seed)
    live = F["m"] > 0
    return {f: rng.normal(size=F[f].shape) * live.reshape(live.shape + (1,) * (F[f].ndim - 3))}


def _adjoint(case, W, with_mass=False):
    """deposit_fields forward and backward on the GPU: fields, dL/dpos, dL/dvel, dL/dmass."""
    import torch

    from pypsi_b200.autograd import deposit_fields

    pos = torch.from_numpy(np.ascontiguousarray(case["pos"].reshape(-1, 3))).cuda().requires_grad_(True)
    vel = torch.from_numpy(np.ascontiguousarray(case["vel"].reshape(-1, 3))).cuda().requires_grad_(True)
    mass = None
    if case["mass"] is not None:
        mass = torch.from_numpy(np.ascontiguousarray(np.asarray(case["mass"], dtype=np.float64).reshape(-1))).cuda()
        mass.requires_grad_(with_mass)
    kw = dict(n=case["n"], bounds=case["bounds"], periodic_box=case["periodic_box"], fields=ALL,
              refine_tolerance=case.get("reftol", 1.0), refine_max_lvl=case.get("maxlvl", 0))
    if case["kind"] == "block":
        kw["block_dims"] = case["pos"].shape[:3]
    else:
        kw["connectivity"] = torch.from_numpy(np.ascontiguousarray(case["conn"], dtype=np.int32)).cuda()
    F = deposit_fields(pos, vel, mass, **kw)
    L = sum((torch.from_numpy(w).cuda() * F[f]).sum() for f, w in W.items())
    L.backward()
    out = {f: t.detach().cpu().numpy() for f, t in F.items()}
    gm = mass.grad.cpu().numpy() if (mass is not None and with_mass) else None
    return out, pos.grad.cpu().numpy(), vel.grad.cpu().numpy(), gm


def _elements(case, p):
    if case["kind"] == "block":
        return block_elements_of(p, case["pos"].shape[:3], case["periodic_box"] is not None)
    return np.nonzero((case["conn"] == p).any(axis=1))[0]


def _check(oracle, case, f, ncoord, seed):
    kind = _kind(oracle)
    conn = cases.conn_of(case)
    ref = cases.run_oracle(oracle, dict(case, fields=ALL), kind=kind)
    W = _weights(ref, f, seed)
    F, gp, gv, _ = _adjoint(case, W)
    for k in ref:  # the forward pass is the reference's deposit, bit for bit
        assert np.array_equal(F[k], ref[k]), k
    rng = np.random.default_rng(seed + 1)
    worst = {}
    for what, g in (("pos", gp), ("vel", gv)):
        if what == "vel" and f in ("m", "x", "xx"):
            assert np.abs(g).max() == 0.0, (f, "depends on no velocity")
            continue
        live = np.nonzero(np.abs(g).sum(axis=1) > 0)[0]
        assert len(live) > 0, (f, what)
        ps = rng.choice(live, size=min(ncoord, len(live)), replace=False)
        axes = rng.integers(0, 3, size=len(ps))
        scale = np.abs(g).max()
        err = 0.0
        for p, ax in zip(ps, axes):
            fd = fd_grad(oracle, kind, case, conn, ref, W, int(p), int(ax), _elements(case, p), what)
            err = max(err, abs(fd - g[p, ax]))
        worst[what] = err / scale
        assert worst[what] <= RTOL, (f, what, worst[what])
    return worst


@pytest.mark.parametrize("field", ["m", "x", "v", "xx", "xv", "vv"])
def test_adjoint_fields_block_mesh_vs_reference_fd(gpu, oracle, field):
    """A 12^3 Zel'dovich lattice (rms 1 cell, velocities 10 psi) on a 24^3 grid in its periodic box."""
    from pypsi_b200.synth import zeldovich

    pos, vel = zeldovich(12, 1.0, 501)
    _check(oracle, cases._block(pos, vel, 24, ALL), field, 24, 7)


@pytest.mark.parametrize("field", ["m", "x", "v", "xx", "xv", "vv"])
def test_adjoint_fields_shell_crossed_subwindow(gpu, oracle, field):
    """Folded sheets (rms 2 cells) on a window inside the periodic box: images and window planes."""
    _check(oracle, cases.make("subwindow"), field, 16, 8)


@pytest.mark.parametrize("field", ["xx", "xv", "vv"])
def test_adjoint_fields_simplex_masses(gpu, oracle, field):
    """Simplex elements with random masses clipped by the grid window; element-mass
    gradients against the deposit of each element alone."""
    case = cases.make("tets")
    _check(oracle, case, field, 16, 9)
    kind = _kind(oracle)
    conn = cases.conn_of(case)
    ref = cases.run_oracle(oracle, dict(case, fields=ALL), kind=kind)
    W = _weights(ref, field, 10)
    _, _, _, gm = _adjoint(case, W, with_mass=True)
    r = ref["x"]
    s = ref["v"]
    R = raw_sums(ref, r, s)
    rng = np.random.default_rng(3)
    for e in rng.choice(conn.shape[0], 8, replace=False):
        me = float(case["mass"][e])
        b = raw_sums(oracle.voxelize(kind, n=case["n"], bounds=case["bounds"], pos=case["pos"], vel=case["vel"],
                                     conn=conn[[e]], mass=np.array([me]), fields=ALL), r, s)
        h = 1e-6 * me
        lp = loss(fields_of({k: R[k] + b[k] * (h / me) for k in R}, r, s), W)
        lm = loss(fields_of({k: R[k] - b[k] * (h / me) for k in R}, r, s), W)
        want = (lp - lm) / (2 * h)
        assert abs(gm[e] - want) <= 1e-5 * max(1.0, np.abs(gm).max()), (e, gm[e], want)


def _refined_tets(case):
    """Tets of the forward deposit (the stats of a psib_voxels call with the case's refinement)."""
    import torch

    from pypsi_b200 import capi

    f = {"m": torch.zeros(case["n"], dtype=torch.float64, device="cuda")}
    pos = torch.from_numpy(np.ascontiguousarray(case["pos"].reshape(-1, 3))).cuda()
    kw = dict(refine_tolerance=case["reftol"], refine_max_lvl=case["maxlvl"], periodic_box=case["periodic_box"])
    if case["kind"] == "block":
        kw["block_dims"] = case["pos"].shape[:3]
    else:
        kw["connectivity"] = torch.from_numpy(np.ascontiguousarray(case["conn"], dtype=np.int32)).cuda()
    return capi.voxels_device(f, case["n"], case["bounds"], pos, **kw)["tets"]


@pytest.mark.parametrize("field", ["m", "x", "xx", "xv", "vv"])
def test_adjoint_fields_refined_block_mesh(gpu, oracle, field):
    """Trilinear refinement up to 2 levels (midpoint criterion, 0.2 cells): each refined
    vertex passes its gradient to the 8 element corners with its trilinear weights."""
    from pypsi_b200.synth import zeldovich

    pos, vel = zeldovich(8, 2.0, 106)
    case = cases._block(pos, vel, 16, ALL, reftol=0.2, maxlvl=2)
    assert _refined_tets(case) > 6 * 8 ** 3
    _check(oracle, case, field, 16, 11)


@pytest.mark.parametrize("field", ["m", "xx", "vv"])
def test_adjoint_fields_triquadratic_refined(gpu, oracle, field):
    """27-node elements refined up to 2 levels: the triquadratic (Lagrange) weights of each
    vertex on the element's 27 nodes, element masses included."""
    from test_gpu_triquadratic import _quad_case

    case = _quad_case(ne=4, maxlvl=2, reftol=0.02, seed=5)
    assert _refined_tets(case) > 6 * 4 ** 3
    _check(oracle, case, field, 16, 12)
    kind = _kind(oracle)
    conn = cases.conn_of(case)
    ref = cases.run_oracle(oracle, dict(case, fields=ALL), kind=kind)
    W = _weights(ref, field, 13)
    _, _, _, gm = _adjoint(case, W, with_mass=True)
    r, s = ref["x"], ref["v"]
    R = raw_sums(ref, r, s)
    for e in np.random.default_rng(4).choice(conn.shape[0], 6, replace=False):
        me = float(case["mass"][e])
        b = raw_sums(oracle.voxelize(kind, n=case["n"], bounds=case["bounds"], pos=case["pos"], vel=case["vel"],
                                     conn=conn[[e]], mass=np.array([me]), fields=ALL, reftol=case["reftol"],
                                     maxlvl=case["maxlvl"]), r, s)
        h = 1e-6 * me
        lp = loss(fields_of({k: R[k] + b[k] * (h / me) for k in R}, r, s), W)
        lm = loss(fields_of({k: R[k] - b[k] * (h / me) for k in R}, r, s), W)
        want = (lp - lm) / (2 * h)
        assert abs(gm[e] - want) <= 1e-5 * max(1.0, np.abs(gm).max()), (e, gm[e], want)


def test_adjoint_fields_rejects_bad_arguments(gpu):
    import ctypes as C

    import torch

    from pypsi_b200 import capi, lib

    n = (4, 4, 4)
    x = torch.zeros((8, 3), dtype=torch.float64, device="cuda")
    z = {f: torch.zeros(n + sh, dtype=torch.float64, device="cuda") for f, sh in
         (("m", ()), ("x", (3,)), ("xx", (3, 3)))}
    g = capi.make_grid(n, ((0.0,) * 3, (1.0,) * 3), {"xx": z["xx"].data_ptr()})
    fwd = capi.make_grid(n, ((0.0,) * 3, (1.0,) * 3), {"m": z["m"].data_ptr()})
    m = capi.make_mesh(8, 1, x.data_ptr(), block_dims=(2, 2, 2))
    gp = torch.zeros_like(x)
    o = capi.Options(precision=0, memory=capi.PSIB_DEVICE, device=-1)
    rc = lib.psib_voxels_adjoint_fields(C.byref(g), C.byref(fwd), C.byref(m), 1.0, 0, gp.data_ptr(), None, None,
                                        C.byref(o))
    assert rc == 1 and b"needs the forward field" in lib.psib_last_error()
