"""Many cutouts in one pass (psib_voxels_batch) against one call per cutout.

Cutouts of uneven size, each with its own periodic box, grid and Zel'dovich
lattice, go through one batch call; every cutout's fields must equal those of
its own psib_voxels call -- FP64 bit for bit, and the mixed and FP64-central
paths to 1e-12 (their per-voxel sums run over the same records in the same
order, so in practice bit for bit as well).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cutouts(k, seed, fields=("m",), lo=4, hi=14, refine=False):
    import torch

    from pypsi_b200.synth import zeldovich

    rng = np.random.default_rng(seed)
    out = []
    for b in range(k):
        n = int(rng.integers(lo, hi + 1))
        side = float(rng.uniform(20.0, 120.0))
        box = ((0.0,) * 3, (side,) * 3)
        pos, vel = zeldovich(n, 1.5, seed * 1000 + b, box=side)
        ng = 2 * n if b % 3 else n + 3  # also grids that are no multiple of the lattice
        shapes = {"m": (ng,) * 3, "x": (ng,) * 3 + (3,), "v": (ng,) * 3 + (3,), "xx": (ng,) * 3 + (3, 3),
                  "xv": (ng,) * 3 + (3, 3), "vv": (ng,) * 3 + (3, 3)}
        bounds = box if b % 4 else ((0.1 * side,) * 3, (0.8 * side,) * 3)  # some sub-windows
        out.append(dict(n=(ng,) * 3, bounds=bounds, pos=torch.from_numpy(pos.reshape(-1, 3).copy()).cuda(),
                        vel=torch.from_numpy(vel.reshape(-1, 3).copy()).cuda(), block_dims=(n,) * 3,
                        periodic_box=box, shapes={f: shapes[f] for f in fields}))
    return out


def _run(cutouts, precision, batch, **kw):
    import torch

    from pypsi_b200 import capi

    for c in cutouts:
        c["fields"] = {f: torch.zeros(sh, dtype=torch.float64, device="cuda") for f, sh in c["shapes"].items()}
    if batch:
        st = capi.voxels_batch_device([{k: v for k, v in c.items() if k != "shapes"} for c in cutouts],
                                      precision=precision, **kw)
    else:
        st = {"tets": 0, "fragments": 0}
        for c in cutouts:
            s1 = capi.voxels_device(c["fields"], c["n"], c["bounds"], c["pos"], c["vel"], block_dims=c["block_dims"],
                                    periodic_box=c["periodic_box"], precision=precision, **kw)
            for k in st:
                st[k] += s1[k]
    torch.cuda.synchronize()
    return [{f: t.cpu().numpy() for f, t in c["fields"].items()} for c in cutouts], st


@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp64-central"])
def test_batch_equals_separate_calls(gpu, precision):
    cutouts = _cutouts(24, 7)
    single, st1 = _run(cutouts, precision, False)
    batch, st = _run(cutouts, precision, True)
    # the same work: tets of the elements each window keeps, and fragments
    assert st["tets"] == st1["tets"] and st["fragments"] == st1["fragments"]
    for b, (s, t) in enumerate(zip(single, batch)):
        assert s["m"].sum() > 0
        if precision == "fp64":
            assert np.array_equal(s["m"], t["m"]), b
        else:
            assert np.abs(s["m"] - t["m"]).max() <= 1e-12 * s["m"].max(), b


def test_batch_all_fields_and_refinement(gpu):
    cutouts = _cutouts(9, 11, fields=("m", "x", "v", "xx", "xv", "vv"), lo=4, hi=8)
    kw = dict(refine_tolerance=0.2, refine_max_lvl=1)
    single, _ = _run(cutouts, "fp64", False, **kw)
    batch, _ = _run(cutouts, "fp64", True, **kw)
    for b, (s, t) in enumerate(zip(single, batch)):
        for f in s:
            assert np.array_equal(s[f], t[f]), (b, f)


def test_batch_rejects_mismatched_fields_and_host_memory(gpu):
    import ctypes as C

    import torch

    from pypsi_b200 import capi, lib

    cutouts = _cutouts(2, 3)
    cutouts[1]["shapes"]["x"] = cutouts[1]["n"] + (3,)
    for c in cutouts:
        c["fields"] = {f: torch.zeros(sh, dtype=torch.float64, device="cuda") for f, sh in c["shapes"].items()}
    with pytest.raises(capi.PsibError, match="same fields"):
        capi.voxels_batch_device([{k: v for k, v in c.items() if k != "shapes"} for c in cutouts])
    o = capi.Options(precision=0, memory=capi.PSIB_HOST, device=-1)
    g = (capi.Grid * 1)()
    m = (capi.Mesh * 1)()
    assert lib.psib_voxels_batch(g, m, 1, 0, 1.0, 0, C.byref(o)) == 6  # PSIB_ERR_UNSUPPORTED
    assert b"device memory" in lib.psib_last_error()


def test_autotune_batch_picks_a_candidate_and_clears(gpu):
    from pypsi_b200 import capi

    cutouts = _cutouts(6, 5)
    import torch

    for c in cutouts:
        c["fields"] = {f: torch.zeros(sh, dtype=torch.float64, device="cuda") for f, sh in c["shapes"].items()}
    args = [{k: v for k, v in c.items() if k != "shapes"} for c in cutouts]
    tune = capi.autotune_batch(args, candidates=(4096, 1 << 16), repeats=1, tiles=(7, -1))
    assert tune["queue_voxels"] in (4096, 1 << 16) and tune["order_cell_bits"] in (7, -1) and tune["ms"] > 0
    assert all(float(t.abs().max()) == 0.0 for c in cutouts for t in c["fields"].values())
    # a tiny capacity forces many passes and must give the same fields
    ref, _ = _run(cutouts, "mixed", True)
    small, _ = _run(cutouts, "mixed", True, queue_voxels=4096)
    for s, t in zip(ref, small):
        assert np.abs(s["m"] - t["m"]).max() <= 1e-12 * s["m"].max()
