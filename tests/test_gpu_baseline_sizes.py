"""Parity at the sizes of the measured workloads, against the reference's own C
code (oracle/_ref, compiled from its sources; the pinned restatement where it
is absent) -- not against this library's other precisions.

* 128^3 particles -> 256^3 voxels, all order-2 fields (the headline workload,
  the bench's own lattice): sixteen-cubed-element sub-blocks of the lattice,
  those that wrap the periodic box included, each on a window of the 256^3
  grid that covers it, and the bench's CPU-baseline sample (window slab 0 of
  16 along x, the whole mesh given, the wrap at x = 0 included).  FP64 equals
  the reference bit for bit; mixed is within 1e-5 of the exact result (the
  oracle in quad precision) and of the reference within 1e-5 plus the
  reference's own rounding.
* 64^3 particles (rms 1 cell) -> 128^3 voxels, density loss: the adjoint's
  gradient at 256 random (particle, axis) coordinates against central finite
  differences (h = 1e-6) of the reference's deposit.
* 256^3 particles (rms 3 cells) -> 512^3 voxels, m and v, refinement up to 2
  levels with the reference's own midpoint criterion (src/refine.c:245-254):
  sampled windows bit for bit against the reference in FP64, total mass
  256^3 to 1e-13 over the whole grid in FP64 and mixed.
* 512 uneven cutouts in one batch call: a seeded sample of them against the
  reference (FP64 bit for bit) and against the exact oracle (mixed, 1e-5).
"""
import math
import multiprocessing as mp
import os

import numpy as np
import pytest

from fd import block_elements_of, fd_loss_grad
from pypsi_b200.metrics import error_maps, field_errors, mass_error

pytestmark = pytest.mark.gpu

BOX = ((0.0,) * 3, (100.0,) * 3)
ALL = ["x", "v", "xx", "xv", "vv"]
MIXED_TOL = 1e-5
MASS_TOL = 1e-13


def _kind(O):
    return "reference" if O.available("reference") else "restatement"


def _check_mixed(out, ref, ex, tol, name):
    """Within tol of the exact result; within tol plus the reference's own
    error of the reference, voxel by voxel."""
    errs = field_errors(out, ex)
    assert errs["m"]["rel"] <= tol, (name, errs["m"])
    for f, e in errs.items():
        if f != "dead_m":
            assert e["norm"] <= tol, (name, f, e)
    e_or = error_maps(out, ref, scale_from=ex)
    e_rx = error_maps(ref, ex)
    for f in e_or:
        bad = e_or[f] > tol + e_rx[f]
        assert not bad.any(), (name, f, float(e_or[f][bad].max()))


# ---------------------------------------------------------------- 128^3 -> 256^3
N2, G2 = 128, 256
_C2 = {}


def _c2():
    if not _C2:
        import oracle as O
        from pypsi_b200.synth import zeldovich

        pos, vel = zeldovich(N2, 2.0, 1234)  # the bench's lattice (rank 0)
        _C2.update(pos=np.ascontiguousarray(pos.reshape(-1, 3)), vel=np.ascontiguousarray(vel.reshape(-1, 3)),
                   conn=O.block_connectivity((N2,) * 3, True))
    return _C2


# sub-block origins: the first two and the last wrap the periodic box on every axis
C2_BLOCKS = [(0, 0, 0), (112, 112, 112), (112, 48, 0), (48, 112, 64), (64, 64, 64), (16, 80, 32), (96, 0, 112),
             (32, 32, 96)]


def block_case(origin, edge=16):
    """The elements of one sub-block of the lattice (periodic connectivity) and
    a window of the 256^3 grid around them: the block's particles unwrapped
    about their median on each axis (so that most of the block lies inside the
    box, where the reference makes its periodic images), padded by one voxel,
    on the grid's planes."""
    c = _c2()
    i, j, k = np.meshgrid(*(np.arange(o, o + edge) for o in origin), indexing="ij")
    elems = (N2 * N2 * i + N2 * j + k).reshape(-1)
    conn = c["conn"][elems]
    p = c["pos"][np.unique(conn)]
    ctr = np.median(p, axis=0)
    L = BOX[1][0]
    pu = p - L * np.round((p - ctr) / L)
    d = L / G2
    lo = np.floor(pu.min(axis=0) / d) - 1
    hi = np.ceil(pu.max(axis=0) / d) + 1
    return dict(conn=conn, n=tuple(int(v) for v in hi - lo), bounds=(tuple(lo * d), tuple(hi * d)))


def _oracle_block(args):
    origin, kind = args
    import oracle as O

    b = block_case(origin)
    c = _c2()
    return origin, O.voxelize(kind, n=b["n"], bounds=b["bounds"], pos=c["pos"], vel=c["vel"], conn=b["conn"],
                              periodic_box=BOX, fields=ALL)


def _psi_run(psi, pos, vel, conn, n, bounds, fields, precision, reftol=1.0, maxlvl=0, mass=None):
    mk = dict(loader="array", pos=pos, vel=vel, connectivity=conn, periodic_box=BOX)
    if mass is not None:
        mk["mass"] = mass
    mesh = psi.Mesh(**mk)
    grid = psi.Grid(type="cart", n=n, bounds=bounds, fields=fields)
    psi.voxels(grid=grid, mesh=mesh, precision=precision, refine_tolerance=reftol, refine_max_lvl=maxlvl)
    return {k: np.array(v) for k, v in grid.fields.items()}


@pytest.fixture(scope="module")
def c2_oracle(oracle):
    """The reference and the exact oracle on every sub-block, on a spawn pool
    (started before this module's first GPU call)."""
    kind = _kind(oracle)
    jobs = [(o, kind) for o in C2_BLOCKS] + [(o, "exact") for o in C2_BLOCKS]
    with mp.get_context("spawn").Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
        res = pool.map(_oracle_block, jobs, chunksize=1)
    ref = dict(res[:len(C2_BLOCKS)])
    ex = dict(res[len(C2_BLOCKS):])
    return ref, ex


def test_c2_blocks_wrap_the_box():
    """The sample includes sub-blocks whose elements cross the periodic box."""
    wrapped = 0
    for o in C2_BLOCKS:
        b = block_case(o)
        wrapped += any(b["bounds"][0][a] < 0.0 or b["bounds"][1][a] > 100.0 for a in range(3))
    assert wrapped >= 3


@pytest.mark.parametrize("origin", C2_BLOCKS)
def test_c2_subblock_fp64_bitwise_and_mixed(gpu, c2_oracle, origin):
    ref, ex = c2_oracle[0][origin], c2_oracle[1][origin]
    b = block_case(origin)
    c = _c2()
    assert ref["m"].sum() > 0.9 * 16 ** 3  # the window holds the block's deposit
    out = _psi_run(gpu, c["pos"], c["vel"], b["conn"], b["n"], b["bounds"], ALL, "fp64")
    for f in ref:
        assert np.array_equal(out[f], ref[f]), (origin, f, float(np.abs(out[f] - ref[f]).max()))
    out = _psi_run(gpu, c["pos"], c["vel"], b["conn"], b["n"], b["bounds"], ALL, "mixed")
    _check_mixed(out, ref, ex, MIXED_TOL, f"c2 block {origin}")


def test_c2_window_slab_fp64_bitwise_and_mixed(gpu, oracle):
    """The bench's CPU-baseline sample: window slab 0 of 16 along x of the
    256^3 grid (16 voxel planes, the periodic wrap at x = 0), every element of
    the mesh given, all fields.  FP64 bit for bit against the reference; mixed
    within 1e-5 of the reference plus the reference's rounding, which is
    estimated by its distance to the FP64-central result (itself within 1e-9
    of the exact oracle on every small parity case)."""
    c = _c2()
    d = BOX[1][0] / G2
    n = (G2 // 16, G2, G2)
    bounds = ((0.0, 0.0, 0.0), (n[0] * d, 100.0, 100.0))
    ref = oracle.voxelize(_kind(oracle), n=n, bounds=bounds, pos=c["pos"], vel=c["vel"], conn=c["conn"],
                          periodic_box=BOX, fields=ALL)
    out = _psi_run(gpu, c["pos"], c["vel"], c["conn"], n, bounds, ALL, "fp64")
    for f in ref:
        assert np.array_equal(out[f], ref[f]), (f, float(np.abs(out[f] - ref[f]).max()))
    cen = _psi_run(gpu, c["pos"], c["vel"], c["conn"], n, bounds, ALL, "fp64-central")
    mix = _psi_run(gpu, c["pos"], c["vel"], c["conn"], n, bounds, ALL, "mixed")
    e_mr = error_maps(mix, ref, scale_from=cen)
    e_rc = error_maps(ref, cen)
    for f in e_mr:
        bad = e_mr[f] > MIXED_TOL + e_rc[f]
        assert not bad.any(), (f, float(e_mr[f][bad].max()))
    assert field_errors(mix, cen)["m"]["rel"] <= MIXED_TOL


# ---------------------------------------------------------------- 64^3 -> 128^3 adjoint
def test_c4_adjoint_256_coordinates_vs_reference_fd(gpu, oracle):
    """64^3 particles (rms 1 cell) on 128^3 voxels, L = sum (m/dV - rho_t)^2
    with rho_t from positions moved by N(0, 0.05 cell): the adjoint's dL/dx at
    256 random (particle, axis) coordinates against central differences of the
    reference's deposit (h = 1e-6), each moving one particle and re-depositing
    the elements around it (the deposit is linear in the tets)."""
    import torch

    from pypsi_b200.autograd import deposit_density
    from pypsi_b200.synth import zeldovich

    n, ng = 64, 128
    pos, _ = zeldovich(n, 1.0, 4321)
    pos = np.ascontiguousarray(pos.reshape(-1, 3))
    dv = (100.0 / ng) ** 3
    kw = dict(n=(ng,) * 3, bounds=BOX, block_dims=(n,) * 3, periodic_box=BOX)
    rng = np.random.default_rng(44)
    tpos = pos + rng.normal(0.0, 0.05 * 100.0 / n, pos.shape)
    with torch.no_grad():
        rho_t = (deposit_density(torch.from_numpy(tpos).cuda(), **kw) / dv).cpu().numpy()
    x = torch.from_numpy(pos.copy()).cuda().requires_grad_(True)
    rho = deposit_density(x, **kw) / dv
    ((rho - torch.from_numpy(rho_t).cuda()) ** 2).sum().backward()
    g = x.grad.cpu().numpy()
    rho = rho.detach().cpu().numpy()
    conn = oracle.block_connectivity((n,) * 3, True)
    case = dict(n=(ng,) * 3, bounds=BOX, pos=pos, mass=None, periodic_box=BOX)
    ps = rng.choice(n ** 3, 256, replace=False)
    axes = rng.integers(0, 3, 256)
    scale = float(np.abs(g).max())
    worst = 0.0
    for p, ax in zip(ps, axes):
        elems = block_elements_of(int(p), (n,) * 3, True)
        fd = fd_loss_grad(oracle, _kind(oracle), case, conn, rho, rho_t, int(p), int(ax), elems)
        worst = max(worst, abs(fd - g[p, ax]))
    assert worst <= 1e-6 * scale, (worst, scale)


# ---------------------------------------------------------------- 256^3 -> 512^3, midpoint refinement
# the midpoint tolerance in voxels: the lattice is smooth at the cell scale (the median face twist of an
# element is a quarter of a voxel), so 0.3 refines about a quarter of the elements once
N5, G5, RT5 = 256, 512, 0.3


@pytest.fixture(scope="module")
def c5_mesh(oracle):
    from pypsi_b200.synth import zeldovich

    pos, vel = zeldovich(N5, 3.0, 5555)
    return (np.ascontiguousarray(pos.reshape(-1, 3)), np.ascontiguousarray(vel.reshape(-1, 3)),
            oracle.block_connectivity((N5,) * 3, True))


C5_WINDOWS = [((0, 0, 0), 24), ((250, 130, 500), 24), ((500, 500, 8), 20)]


@pytest.mark.parametrize("win", C5_WINDOWS)
def test_c5_midpoint_refinement_windows_bitwise(gpu, oracle, c5_mesh, win):
    """Windows of the 512^3 grid (some at the box faces), the whole 256^3 mesh
    given, refinement to 2 levels where a trilinear edge midpoint deviates by
    more than 0.3 voxel (the reference's criterion): FP64 bit for bit."""
    pos, vel, conn = c5_mesh
    (i0, j0, k0), w = win
    d = 100.0 / G5
    n = (w, w, w)
    bounds = ((i0 * d, j0 * d, k0 * d), ((i0 + w) * d, (j0 + w) * d, (k0 + w) * d))
    ref = oracle.voxelize(_kind(oracle), n=n, bounds=bounds, pos=pos, vel=vel, conn=conn, periodic_box=BOX,
                          fields=["v"], reftol=RT5, maxlvl=2)
    assert ref["m"].sum() > 0
    out = _psi_run(gpu, pos, vel, conn, n, bounds, ["v"], "fp64", reftol=RT5, maxlvl=2)
    for f in ref:
        assert np.array_equal(out[f], ref[f]), (win, f, float(np.abs(out[f] - ref[f]).max()))


def test_c5_midpoint_refinement_full_mass(gpu, c5_mesh):
    """The whole 512^3 grid, m and v, midpoint refinement to 2 levels: total
    mass 256^3 to 1e-13 relative, FP64 and mixed."""
    import torch

    from pypsi_b200 import capi

    pos, vel, _ = c5_mesh
    dpos = torch.from_numpy(pos).cuda()
    dvel = torch.from_numpy(vel).cuda()
    for prec in ("fp64", "mixed"):
        f = {"m": torch.zeros((G5,) * 3, dtype=torch.float64, device="cuda"),
             "v": torch.zeros((G5,) * 3 + (3,), dtype=torch.float64, device="cuda")}
        st = capi.voxels_device(f, (G5,) * 3, BOX, dpos, dvel, block_dims=(N5,) * 3, periodic_box=BOX,
                                precision=prec, refine_tolerance=RT5, refine_max_lvl=2)
        assert st["tets"] > 6 * N5 ** 3  # the criterion refined something
        merr = mass_error(f["m"].cpu().numpy(), N5 ** 3)
        assert merr <= MASS_TOL, (prec, merr)
        del f
    capi.lib.psib_release_device_memory()


# ---------------------------------------------------------------- 512 cutouts in one batch
def _c3_cutouts():
    """The bench's 512 cutouts: edge n log-uniform in [8, 64] (seed 333), each a
    Zel'dovich lattice (rms 1.5 cells) in its own periodic box of side 100 on a
    (2n)^3 grid."""
    from pypsi_b200.synth import zeldovich

    rng = np.random.default_rng(333)
    ns = [int(round(math.exp(rng.uniform(math.log(8), math.log(64))))) for _ in range(512)]
    return [(n,) + zeldovich(n, 1.5, 10000 + b) for b, n in enumerate(ns)]


def _oracle_cutout(args):
    n, pos, kind = args
    import oracle as O

    return O.voxelize(kind, n=(2 * n,) * 3, bounds=BOX, pos=pos.reshape(-1, 3),
                      conn=O.block_connectivity((n,) * 3, True), periodic_box=BOX)


def test_c3_batch_sample_against_reference(gpu, oracle):
    import torch

    from pypsi_b200 import capi

    cuts = _c3_cutouts()
    rng = np.random.default_rng(3)
    # a seeded sample: 12 cutouts up to n = 40 for FP64 (reference time), 6 up to n = 14 for the exact oracle
    fp64_idx = [int(i) for i in rng.permutation(512) if cuts[i][0] <= 40][:12]
    mix_idx = [int(i) for i in rng.permutation(512) if cuts[i][0] <= 14][:6]
    jobs = [(cuts[i][0], cuts[i][1], _kind(oracle)) for i in fp64_idx] + \
           [(cuts[i][0], cuts[i][1], "exact") for i in mix_idx] + \
           [(cuts[i][0], cuts[i][1], _kind(oracle)) for i in mix_idx]
    with mp.get_context("spawn").Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
        res = pool.map(_oracle_cutout, jobs, chunksize=1)
    ref64 = res[:len(fp64_idx)]
    ex = res[len(fp64_idx):len(fp64_idx) + len(mix_idx)]
    refm = res[len(fp64_idx) + len(mix_idx):]

    def batch(precision):
        cut = []
        for n, pos, _ in cuts:
            cut.append(dict(n=(2 * n,) * 3, bounds=BOX, pos=torch.from_numpy(pos.reshape(-1, 3).copy()).cuda(),
                            block_dims=(n,) * 3, periodic_box=BOX,
                            fields={"m": torch.zeros((2 * n,) * 3, dtype=torch.float64, device="cuda")}))
        capi.voxels_batch_device(cut, precision=precision)
        torch.cuda.synchronize()
        return cut

    cut = batch("fp64")
    for i, r in zip(fp64_idx, ref64):
        assert np.array_equal(cut[i]["fields"]["m"].cpu().numpy(), r["m"]), (i, cuts[i][0])
    del cut
    cut = batch("mixed")
    for i, e, r in zip(mix_idx, ex, refm):
        _check_mixed({"m": cut[i]["fields"]["m"].cpu().numpy()}, r, e, MIXED_TOL, f"cutout {i}")
    for c in cut:
        n = round(c["n"][0] / 2)
        assert mass_error(c["fields"]["m"].cpu().numpy(), n ** 3) <= MASS_TOL
    del cut
    capi.lib.psib_release_device_memory()
