"""Adjoint of the density deposit (psib_voxels_adjoint via torch.autograd).

The loss is L = sum (m / dV - rho_target)^2.  Its gradient with respect to
particle positions, from the adjoint kernel, is checked against central finite
differences (h = 1e-6) of the reference's own C path (oracle/_ref when it was
built, else the restatement that is pinned to it) and of this library's FP64
forward pass, on seeded random coordinates.  The finite differences move one
particle and re-deposit only the elements that contain it (the deposit is
linear in the tets).  Mass gradients are checked against the deposit of each
element alone, and at 64^3 particles -> 128^3 voxels a directional derivative
over all particles is checked against the forward pass.
"""
import numpy as np
import pytest

import cases
from fd import block_elements_of, fd_loss_grad

pytestmark = pytest.mark.gpu

# |adjoint - finite difference| <= RTOL * max |gradient| (the finite differences
# themselves are good to ~1e-8 of that scale in FP64 at h = 1e-6)
RTOL = 1e-6


def _ref_kind(O):
    return "reference" if O.available("reference") else "restatement"


def _setup(case, target_sigma_cells=0.05, seed=5):
    import torch

    from pypsi_b200.autograd import deposit_density

    n, bounds = case["n"], case["bounds"]
    dv = float(np.prod([(bounds[1][i] - bounds[0][i]) / n[i] for i in range(3)]))
    pos = np.array(case["pos"], dtype=np.float64).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    cell = (bounds[1][0] - bounds[0][0]) / n[0]
    tpos = pos + rng.normal(0.0, target_sigma_cells * cell, pos.shape)
    kw = dict(n=n, bounds=bounds, periodic_box=case["periodic_box"], refine_tolerance=case.get("reftol", 1.0),
              refine_max_lvl=case.get("maxlvl", 0))
    if case["kind"] == "block":
        kw["block_dims"] = case["pos"].shape[:3]
    else:
        kw["connectivity"] = torch.from_numpy(np.ascontiguousarray(case["conn"], dtype=np.int32)).cuda()
    mass = None if case["mass"] is None else torch.from_numpy(np.asarray(case["mass"], dtype=np.float64).reshape(-1)).cuda()
    with torch.no_grad():
        rho_t = deposit_density(torch.from_numpy(tpos).cuda(), mass, **kw) / dv
    x = torch.from_numpy(pos.copy()).cuda().requires_grad_(True)
    if mass is not None:
        mass = mass.clone().requires_grad_(True)
    m = deposit_density(x, mass, **kw)
    rho = m / dv
    loss = ((rho - rho_t) ** 2).sum()
    loss.backward()
    return dict(pos=pos, x=x, mass=mass, rho=rho.detach().cpu().numpy(), rho_t=rho_t.cpu().numpy(), dv=dv, kw=kw,
                grad=x.grad.cpu().numpy(), loss=float(loss))


def _elements(case, p):
    if case["kind"] == "block":
        return block_elements_of(p, case["pos"].shape[:3], case["periodic_box"] is not None)
    return np.nonzero((case["conn"] == p).any(axis=1))[0]


def _check_fd(oracle, case, s, kinds, ncoord, seed=11):
    conn = cases.conn_of(case)
    g = s["grad"]
    rng = np.random.default_rng(seed)
    npart = g.shape[0]
    # sample particles that have a gradient (some tets of small cases never reach the window)
    live = np.nonzero(np.abs(g).sum(axis=1) > 0)[0]
    assert len(live) > 0
    ps = rng.choice(live, size=min(ncoord, len(live)), replace=False)
    axes = rng.integers(0, 3, size=len(ps))
    scale = np.abs(g).max()
    worst = {}
    for kind in kinds:
        err = 0.0
        for p, ax in zip(ps, axes):
            fd = fd_loss_grad(oracle, kind, case, conn, s["rho"], s["rho_t"], int(p), int(ax), _elements(case, p))
            err = max(err, abs(fd - g[p, ax]))
        worst[kind] = err / scale
    assert all(v <= RTOL for v in worst.values()), (worst, npart)
    return worst


def test_adjoint_block_mesh_vs_reference_fd(gpu, oracle):
    """A 16^3 Zel'dovich lattice (rms 1 cell) on a 32^3 grid, the shape of the
    64^3 -> 128^3 differentiable workload: 96 coordinates."""
    from pypsi_b200.synth import zeldovich

    pos, vel = zeldovich(16, 1.0, 401)
    case = cases._block(pos, vel, 32, [])
    s = _setup(case)
    _check_fd(oracle, case, s, [_ref_kind(oracle), "restatement"], 96)


def test_adjoint_shell_crossed_subwindow(gpu, oracle):
    """Folded sheets (rms 2 cells), a window inside the periodic box: periodic
    images and window planes (which do not move with the particles)."""
    case = cases.make("subwindow")
    case["fields"] = []
    s = _setup(case)
    _check_fd(oracle, case, s, [_ref_kind(oracle)], 64)


def test_adjoint_simplex_elements_with_masses(gpu, oracle):
    """Simplex elements ('array' loader) with random masses, clipped by the grid window."""
    case = cases.make("tets")
    case["fields"] = []
    s = _setup(case)
    _check_fd(oracle, case, s, [_ref_kind(oracle)], 64)
    # dL/dmass_e = sum_v dL/drho_v * rho_e,v / mass_e (the deposit is linear in the masses)
    gm = s["mass"].grad.cpu().numpy()
    conn = cases.conn_of(case)
    dl = 2.0 * (s["rho"] - s["rho_t"])
    rng = np.random.default_rng(3)
    for e in rng.choice(conn.shape[0], 16, replace=False):
        me = float(case["mass"][e])
        de = oracle.voxelize(_ref_kind(oracle), n=case["n"], bounds=case["bounds"], pos=case["pos"], conn=conn[[e]],
                             mass=np.array([me]), fields=[])["m"] / s["dv"]
        want = float(np.sum(dl * de)) / me
        assert abs(gm[e] - want) <= 1e-10 * max(1.0, abs(want)), (e, gm[e], want)


def test_adjoint_nonperiodic_block_with_masses(gpu, oracle):
    case = cases.make("nonperiodic")
    case["fields"] = []
    s = _setup(case)
    _check_fd(oracle, case, s, [_ref_kind(oracle)], 48)


def test_adjoint_refined_block_mesh(gpu, oracle):
    """Trilinear refinement up to 2 levels (midpoint criterion, tolerance 0.2 cells): the
    gradient flows to the element corners through the trilinear weights of each refined vertex."""
    case = cases.make("refine")
    case["fields"] = []
    s = _setup(case)
    _check_fd(oracle, case, s, [_ref_kind(oracle)], 48)


def test_adjoint_zero_inside_one_voxel(gpu):
    """A tet strictly inside one voxel deposits its whole mass there whatever its
    shape: the gradient is zero."""
    import torch

    from pypsi_b200 import capi

    pos = torch.tensor([[0.31, 0.32, 0.33], [0.36, 0.33, 0.34], [0.32, 0.37, 0.35], [0.33, 0.34, 0.38]],
                       dtype=torch.float64, device="cuda")
    conn = torch.arange(4, dtype=torch.int32, device="cuda").reshape(1, 4)
    gm = torch.rand((4, 4, 4), dtype=torch.float64, device="cuda")
    gp = torch.zeros_like(pos)
    gmass = torch.zeros(1, dtype=torch.float64, device="cuda")
    capi.adjoint_device(gm, (4, 4, 4), ((0.0,) * 3, (1.0,) * 3), pos, gp, connectivity=conn, grad_mass=gmass)
    # the moving faces sum to dS(T)/dx_i and cancel against m0 dS(T)/dx_i, up to
    # rounding at the scale g * area / volume (~ 40 here)
    assert float(gp.abs().max()) <= 1e-12
    assert abs(float(gmass[0]) - float(gm[1, 1, 1])) <= 1e-15


def test_adjoint_is_linear_and_accumulates(gpu):
    import torch

    from pypsi_b200 import capi
    from pypsi_b200.synth import zeldovich

    pos, _ = zeldovich(16, 2.0, 402)
    box = cases.BOX
    x = torch.from_numpy(pos.reshape(-1, 3).copy()).cuda()
    n = (32, 32, 32)
    g1 = torch.randn(n, dtype=torch.float64, device="cuda")
    g2 = torch.randn(n, dtype=torch.float64, device="cuda")

    def adj(g, out=None):
        out = torch.zeros_like(x) if out is None else out
        capi.adjoint_device(g, n, box, x, out, block_dims=(16, 16, 16), periodic_box=box)
        return out

    a, b = adj(g1), adj(g2)
    c = adj(2.0 * g1 - 3.0 * g2)
    assert float((c - (2.0 * a - 3.0 * b)).abs().max()) <= 1e-11 * float(c.abs().max())
    acc = adj(g2, adj(g1))  # accumulates into the given buffer
    assert float((acc - (a + b)).abs().max()) <= 1e-12 * float(acc.abs().max())


def test_adjoint_rejects_unsupported(gpu):
    import torch

    from pypsi_b200 import capi, lib

    x = torch.zeros((8, 3), dtype=torch.float64, device="cuda")
    g = capi.make_grid((4, 4, 4), ((0.0,) * 3, (1.0,) * 3), {"m": torch.zeros((4, 4, 4), dtype=torch.float64,
                                                                               device="cuda").data_ptr()})
    m = capi.make_mesh(8, 1, x.data_ptr(), block_dims=(2, 2, 2))
    gp = torch.zeros_like(x)
    o = capi.Options(precision=0, memory=capi.PSIB_DEVICE, device=-1)
    import ctypes as C

    z = torch.zeros((4, 4, 4, 3), dtype=torch.float64, device="cuda")
    zm = torch.zeros((4, 4, 4), dtype=torch.float64, device="cuda")
    gx = capi.make_grid((4, 4, 4), ((0.0,) * 3, (1.0,) * 3), {"m": zm.data_ptr(), "x": z.data_ptr()})
    rc = lib.psib_voxels_adjoint(C.byref(gx), C.byref(m), 1.0, 0, gp.data_ptr(), None, None, C.byref(o))
    assert rc == 6 and b"field m only" in lib.psib_last_error()


def test_adjoint_directional_derivative_64cube_to_128cube(gpu):
    """The differentiable workload at full size: 64^3 particles (rms 1 cell)
    onto 128^3 voxels.  g . d against (L(x + eps d) - L(x - eps d)) / 2 eps of
    the FP64 forward pass, over all particles at once."""
    import torch

    from pypsi_b200.autograd import deposit_density
    from pypsi_b200.synth import zeldovich

    pos, _ = zeldovich(64, 1.0, 403)
    case = cases._block(pos, None, 128, [])
    s = _setup(case)
    d = torch.from_numpy(np.random.default_rng(9).normal(size=s["pos"].shape)).cuda()
    eps = 1e-7
    x0 = torch.from_numpy(s["pos"]).cuda()
    rho_t = torch.from_numpy(s["rho_t"]).cuda()

    def loss(x):
        with torch.no_grad():
            return float(((deposit_density(x, **s["kw"]) / s["dv"] - rho_t) ** 2).sum())

    fd = (loss(x0 + eps * d) - loss(x0 - eps * d)) / (2 * eps)
    gd = float((torch.from_numpy(s["grad"]).cuda() * d).sum())
    assert abs(fd - gd) <= 1e-4 * abs(gd), (fd, gd)
