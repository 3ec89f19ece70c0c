"""PSI.VDF and PSI.RStarTree on the GPU (psib_sample_vdf, psib_query_elements).

Through the drop-in module, one point or box per call as the reference's API
has it, and through the batched C ABI, many points per call (host and device
memory): the same samples and elements as the oracle, bit for bit and in the
same order (descending element, then tet), and as the compiled reference
wherever its tree is one leaf (at most 32 elements); the same sets beyond."""
import numpy as np
import pytest

import oracle as O
from vdf_cases import LARGE, SMALL, make, sorted_samples, vdf

pytestmark = pytest.mark.gpu


def module_mesh(PSI, c):
    kw = dict(loader="array", pos=c["pos"], vel=c["vel"], mass=c["mass"], connectivity=c["conn"])
    if c["periodic_box"] is not None:
        kw["periodic_box"] = c["periodic_box"]
    return PSI.Mesh(**kw)


@pytest.mark.parametrize("tree", [False, True])
@pytest.mark.parametrize("name", SMALL + LARGE)
def test_vdf_module(gpu, oracle, name, tree):
    c = make(name)
    mesh = module_mesh(gpu, c)
    t = gpu.RStarTree(mesh) if tree else None
    total = 0
    for p in c["points"]:
        kw = dict(refine_tolerance=c["reftol"], refine_max_lvl=c["maxlvl"])
        rho, vel = gpu.VDF(mesh, tuple(p), t, **kw) if tree else gpu.VDF(mesh, tuple(p), **kw)
        w_rho, w_vel = vdf(c, "restatement", p, tree)
        assert np.array_equal(rho, w_rho) and np.array_equal(vel, w_vel), (name, p)
        total += len(rho)
        if oracle.available("reference"):
            r_rho, r_vel = vdf(c, "reference", p, tree)
            if name in SMALL:
                assert np.array_equal(rho, r_rho) and np.array_equal(vel, r_vel)
            else:
                assert np.array_equal(sorted_samples(rho, vel), sorted_samples(r_rho, r_vel))
    if tree or c["periodic_box"] is not None:
        assert total > 0


@pytest.mark.parametrize("name", SMALL + LARGE)
def test_rstartree_query(gpu, oracle, name):
    c = make(name)
    tree = gpu.RStarTree(module_mesh(gpu, c))
    win = O.tree_window(c["periodic_box"])
    rng = np.random.default_rng(9)
    for _ in range(6):
        lo = rng.uniform(-0.1, 0.9, 3)
        box = (tuple(lo), tuple(lo + rng.uniform(0.0, 0.4, 3)))
        got = tree.query(box)
        assert got.dtype == np.int32
        assert np.array_equal(got, O.query_elements("restatement", c["pos"], c["conn"], win, box, c["periodic_box"]))
        if oracle.available("reference"):
            ref = O.query_elements("reference", c["pos"], c["conn"], win, box, c["periodic_box"])
            assert np.array_equal(got if name in SMALL else np.sort(got), ref if name in SMALL else np.sort(ref))
    with pytest.raises(TypeError, match="two tuples"):
        tree.query((1, 2, 3))


def test_vdf_batched_host_and_device(gpu, oracle):
    """Many points per call through psib_sample_vdf, with refinement."""
    import torch

    from pypsi_b200 import capi

    c = make("periodic5")
    pts = np.random.default_rng(3).uniform(0, 1, (500, 3))
    kw = dict(connectivity=c["conn"], vel=c["vel"], mass=c["mass"], periodic_box=c["periodic_box"],
              refine_tolerance=c["reftol"], refine_max_lvl=c["maxlvl"])
    off, rho, vel = capi.sample_vdf(pts, c["pos"], **kw)
    # the oracle finds 203 samples at these points (stored-position partners leave gaps near the box edge)
    assert off[0] == 0 and off[-1] == len(rho) == 203
    for i in range(0, 500, 3):
        w_rho, w_vel = vdf(c, "restatement", pts[i], True)
        assert np.array_equal(rho[off[i]:off[i + 1]], w_rho), i
        assert np.array_equal(vel[off[i]:off[i + 1]], w_vel), i
    dev = {k: torch.tensor(v, device="cuda") for k, v in (("connectivity", c["conn"]), ("vel", c["vel"]),
                                                             ("mass", c["mass"]))}
    doff, drho, dvel = capi.sample_vdf(torch.tensor(pts, device="cuda"), torch.tensor(c["pos"], device="cuda"),
                                       periodic_box=c["periodic_box"], refine_tolerance=c["reftol"],
                                       refine_max_lvl=c["maxlvl"], **dev)
    torch.cuda.synchronize()
    assert np.array_equal(doff.cpu().numpy(), off)
    assert np.array_equal(drho.cpu().numpy(), rho) and np.array_equal(dvel.cpu().numpy(), vel)


def test_vdf_triquadratic_against_reference(gpu, oracle):
    from test_gpu_triquadratic import _quad_case

    kind = "reference" if oracle.available("reference") else "restatement"

    q = _quad_case(ne=3, maxlvl=1, reftol=0.01)  # 27 elements: one leaf
    mesh = gpu.Mesh(loader="array", pos=q["pos"], vel=q["vel"], mass=q["mass"], connectivity=q["conn"])
    tree = gpu.RStarTree(mesh)
    n = 0
    for p in np.random.default_rng(4).uniform(0.1, 0.9, (10, 3)):
        rho, vel = gpu.VDF(mesh, tuple(p), tree, refine_tolerance=0.01, refine_max_lvl=1)
        r_rho, r_vel = O.sample_vdf(kind, q["pos"], q["conn"], p, vel=q["vel"], mass=q["mass"],
                                    window=O.tree_window(None), reftol=0.01, maxlvl=1)
        assert np.array_equal(rho, r_rho) and np.array_equal(vel, r_vel)
        n += len(rho)
    assert n > 0


def test_vdf_from_block_and_snapshot_loaders(gpu, oracle, tmp_path):
    """Implicit block connectivity and a loaded Gadget-2 snapshot."""
    from snapshots import make_snapshot

    path = str(tmp_path / "snap")
    make_snapshot(path, 6)
    mesh = gpu.Mesh(loader="gadget2", filename=path)
    box = mesh.wrapbox
    for p in ((10.0, 20.0, 30.0), (33.3, 5.5, 17.0)):
        rho, vel = gpu.VDF(mesh, p)
        w_rho, w_vel = O.sample_vdf("restatement", mesh.pos, mesh.connectivity, p, vel=mesh.vel, mass=mesh.mass,
                                    periodic_box=box)
        assert np.array_equal(rho, w_rho) and np.array_equal(vel, w_vel)
    c = make("open4_mild")
    bmesh = gpu.Mesh(loader="block", pos=np.ascontiguousarray(c["pos"].reshape(4, 4, 4, 3)),
                     vel=np.ascontiguousarray(c["vel"].reshape(4, 4, 4, 3)))
    tree = gpu.RStarTree(bmesh)
    for p in c["points"][1:4]:
        rho, vel = gpu.VDF(bmesh, tuple(p), tree)
        w_rho, w_vel = O.sample_vdf("restatement", c["pos"], c["conn"], p, vel=c["vel"], window=O.tree_window(None))
        assert np.array_equal(rho, w_rho) and np.array_equal(vel, w_vel)


def test_index_equals_stateless_calls(gpu, oracle):
    """psib_index_create / _query / _sample_vdf answer as psib_query_elements and
    psib_sample_vdf do, over many points and boxes, and the index outlives the
    caller's arrays (it holds its own copy of the mesh)."""
    import ctypes as C

    from pypsi_b200 import capi

    c = make("periodic5")
    pos, conn, vel, mass = (np.ascontiguousarray(c[k]) for k in ("pos", "conn", "vel", "mass"))
    m = capi.make_mesh(len(pos), len(conn), pos.ctypes.data, vel.ctypes.data, mass.ctypes.data, conn.ctypes.data, 8,
                       None, c["periodic_box"])
    win = np.ascontiguousarray(O.tree_window(c["periodic_box"]), dtype=np.float64)
    lib = capi.lib
    lib.psib_index_create.argtypes = [C.POINTER(capi.Mesh), C.c_void_p, C.POINTER(C.c_void_p), C.c_void_p]
    lib.psib_index_query.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p, C.c_longlong,
                                     C.c_void_p]
    lib.psib_index_sample_vdf.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_double, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p]
    lib.psib_index_destroy.argtypes = [C.c_void_p]
    ix = C.c_void_p()
    assert lib.psib_index_create(C.byref(m), win.ctypes.data, C.byref(ix), None) == 0
    try:
        pos2 = pos.copy()
        pos[:] = 0.0  # the index keeps the mesh as it was
        pts = np.random.default_rng(8).uniform(0, 1, (300, 3))
        want_off, want_rho, want_vel = capi.sample_vdf(pts, pos2, connectivity=conn, vel=vel, mass=mass,
                                                       periodic_box=c["periodic_box"], refine_tolerance=c["reftol"],
                                                       refine_max_lvl=c["maxlvl"])
        off = np.zeros(len(pts) + 1, dtype=np.int64)
        n = int(want_off[-1])
        rho, v = np.zeros(max(n, 1)), np.zeros((max(n, 1), 3))
        assert lib.psib_index_sample_vdf(ix, pts.ctypes.data, len(pts), c["reftol"], c["maxlvl"], off.ctypes.data,
                                         rho.ctypes.data, v.ctypes.data, n, None) == 0
        assert np.array_equal(off, want_off)
        assert np.array_equal(rho[:n], want_rho) and np.array_equal(v[:n], want_vel)
        lo = np.random.default_rng(2).uniform(-0.1, 0.9, (20, 3))
        boxes = np.ascontiguousarray(np.concatenate([lo, lo + 0.3], axis=1))
        qoff = np.zeros(21, dtype=np.int64)
        assert lib.psib_index_query(ix, boxes.ctypes.data, 20, qoff.ctypes.data, None, 0, None) == 0
        els = np.zeros(max(int(qoff[-1]), 1), dtype=np.int32)
        assert lib.psib_index_query(ix, boxes.ctypes.data, 20, qoff.ctypes.data, els.ctypes.data, int(qoff[-1]),
                                    None) == 0
        for b in range(20):
            want = O.query_elements("restatement", pos2, conn, win, (tuple(lo[b]), tuple(lo[b] + 0.3)),
                                    c["periodic_box"])
            assert np.array_equal(els[qoff[b]:qoff[b + 1]], want), b
    finally:
        lib.psib_index_destroy(ix)
