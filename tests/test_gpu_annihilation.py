"""Annihilation mode on the GPU: PSI.voxels(grid, mesh, mode='annihilation').

The GPU visits element pairs in the oracle's order (e ascending, e1
descending), so its m field equals the oracle's bit for bit on every case, and
the reference's wherever the reference's R*-tree is one leaf (at most 32
kept elements); the work counters equal the oracle's.  Also: the device-memory
call, streaming in chunks, accumulation into a filled grid, the implicit block
connectivity and triquadratic elements (against the compiled reference)."""
import numpy as np
import pytest

from ann_cases import LARGE, SMALL, make, run_oracle

pytestmark = pytest.mark.gpu


def run_gpu(PSI, c, m0=None, **kw):
    grid = PSI.Grid(type="cart", n=c["n"], bounds=c["bounds"])
    if m0 is not None:
        grid.fields["m"][...] = m0
    mk = dict(loader="array", pos=np.ascontiguousarray(c["pos"], dtype=np.float64), connectivity=c["conn"])
    if c["mass"] is not None:
        mk["mass"] = np.asarray(c["mass"], dtype=np.float64)
    if c["periodic_box"] is not None:
        mk["periodic_box"] = c["periodic_box"]
    mesh = PSI.Mesh(**mk)
    PSI.voxels(grid=grid, mesh=mesh, mode="annihilation", refine_tolerance=c["reftol"], refine_max_lvl=c["maxlvl"],
               **kw)
    return np.array(grid.fields["m"]), PSI.last_stats()


@pytest.mark.parametrize("name", SMALL + LARGE + ["degenerate"])
def test_annihilation_bitwise(gpu, oracle, name):
    c = make(name)
    want, cnt = run_oracle(c, counters=True)
    got, st = run_gpu(gpu, c)
    assert np.array_equal(got, want["m"], equal_nan=True), (name, np.nanmax(np.abs(got - want["m"])))
    assert st["tet_images"] == cnt["tet_images"]  # tet pairs
    assert st["fragments"] == cnt["fragments"]
    assert st["splits"] == cnt["splits"]
    assert st["elements_kept"] == cnt["elements_kept"]
    if name in SMALL and oracle.available("reference"):
        assert np.array_equal(got, run_oracle(c, "reference")["m"])


def test_annihilation_chunks_and_accumulation(gpu, oracle, monkeypatch):
    c = make("periodic5")
    m0 = np.random.default_rng(7).uniform(0, 100, c["n"])
    want = run_oracle(c)["m"]
    out = {"m": m0.copy()}
    oracle.voxelize("restatement", c["n"], c["bounds"], c["pos"], c["conn"], periodic_box=c["periodic_box"],
                    mode="annihilation", out=out)
    monkeypatch.setenv("PSIB_ANN_BUDGET", "997")  # many chunks of ~1000 tet pairs
    got, st = run_gpu(gpu, c, m0=m0)
    assert st["chunks"] > 10
    assert np.array_equal(got, out["m"])
    monkeypatch.delenv("PSIB_ANN_BUDGET")
    got, st = run_gpu(gpu, c)
    assert st["chunks"] == 1
    assert np.array_equal(got, want)


def test_annihilation_device_memory_and_block_loader(gpu, oracle):
    import torch

    from pypsi_b200 import capi

    c = make("block6")
    want = run_oracle(c)["m"]
    m = torch.zeros(c["n"], dtype=torch.float64, device="cuda")
    capi.voxels_device({"m": m}, c["n"], c["bounds"], torch.tensor(c["pos"], device="cuda"),
                       connectivity=torch.tensor(c["conn"], device="cuda"), mode="annihilation")
    torch.cuda.synchronize()
    assert np.array_equal(m.cpu().numpy(), want)
    # the same lattice through loader='block' (implicit connectivity)
    grid = gpu.Grid(n=c["n"], bounds=c["bounds"])
    mesh = gpu.Mesh(loader="block", pos=np.ascontiguousarray(c["pos"].reshape(6, 6, 6, 3)))
    gpu.voxels(grid=grid, mesh=mesh, mode="annihilation")
    assert np.array_equal(grid.fields["m"], want)


def test_annihilation_triquadratic_against_reference(gpu, oracle):
    from test_gpu_triquadratic import _quad_case

    kind = "reference" if oracle.available("reference") else "restatement"
    for maxlvl, reftol in ((0, 1.0), (1, 0.05)):
        q = _quad_case(ne=3, maxlvl=maxlvl, reftol=reftol)  # 27 elements: one R*-tree leaf
        ref = oracle.voxelize(kind, q["n"], q["bounds"], q["pos"], q["conn"], mass=q["mass"], reftol=reftol,
                              maxlvl=maxlvl, mode="annihilation")["m"]
        c = dict(n=q["n"], bounds=q["bounds"], pos=q["pos"], conn=q["conn"], mass=q["mass"], periodic_box=None,
                 reftol=reftol, maxlvl=maxlvl)
        got, _ = run_gpu(gpu, c)
        assert np.abs(ref).max() > 0
        assert np.array_equal(got, ref), maxlvl


def test_annihilation_rejections(gpu):
    c = make("block3")
    grid = gpu.Grid(n=c["n"], bounds=c["bounds"])
    mesh = gpu.Mesh(loader="array", pos=c["pos"], connectivity=c["conn"])
    with pytest.raises(NotImplementedError, match="midpoint"):
        gpu.voxels(grid=grid, mesh=mesh, mode="annihilation", refine_criterion="stretch", refine_max_lvl=1)
