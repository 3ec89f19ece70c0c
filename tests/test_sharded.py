"""One mesh over several ranks: element slabs and the field exchange.

Each rank of a world-size-2 (and 3) gloo group deposits its slab of elements
with the oracle on the CPU -- standing in for its GPU -- and the ranks combine
their grids with pypsi_b200.parallel.merge_fields, the exchange step that the
multi-GPU path runs over NCCL.  The merged fields must equal the oracle's
deposit of the whole mesh to FP64 rounding (the sums run in another order).
"""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

import cases
from pypsi_b200.metrics import field_errors

TOL = 1e-12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, name, out_dir):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch
    import torch.distributed as dist

    import cases as C
    import oracle as O
    from pypsi_b200.parallel import element_slab, merge_fields

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        c = C.make(name)
        conn = C.conn_of(c)
        e0, e1 = element_slab(conn.shape[0], world, rank)
        mass = None if c["mass"] is None else np.asarray(c["mass"]).reshape(-1)[e0:e1]
        part = O.voxelize("restatement", n=c["n"], bounds=c["bounds"], pos=c["pos"].reshape(-1, 3),
                          vel=c["vel"].reshape(-1, 3), conn=conn[e0:e1], mass=mass, periodic_box=c["periodic_box"],
                          fields=c["fields"], reftol=c["reftol"], maxlvl=c["maxlvl"])
        fields = {k: torch.from_numpy(v) for k, v in part.items()}
        merge_fields(fields)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), **{k: v.numpy() for k, v in fields.items()})
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("c2_small", 2), ("subwindow", 2), ("nonperiodic", 3), ("refine", 2)])
def test_sharded_deposit_matches_single(oracle, tmp_path, name, world):
    import torch.multiprocessing as mp

    mp.start_processes(_worker, args=(world, _free_port(), name, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    ref = cases.run_oracle(oracle, cases.make(name))
    outs = [dict(np.load(os.path.join(tmp_path, f"rank{r}.npz"))) for r in range(world)]
    for r in range(1, world):  # every rank holds the same result
        for f in ref:
            assert np.array_equal(outs[r][f], outs[0][f]), (r, f)
    errs = field_errors(outs[0], ref)
    assert errs["m"]["rel"] <= TOL, errs["m"]
    for f, e in errs.items():
        if f != "dead_m":
            assert e["norm"] <= TOL, (f, e)
    assert errs["dead_m"] == 0.0


def test_slabs_cover_the_mesh_and_match_block_connectivity(oracle):
    import torch

    from pypsi_b200.parallel import block_slab_connectivity, element_slab

    for nelem, world in [(10, 3), (7, 8), (4096, 4)]:
        slabs = [element_slab(nelem, world, r) for r in range(world)]
        assert slabs[0][0] == 0 and slabs[-1][1] == nelem
        assert all(slabs[r][1] == slabs[r + 1][0] for r in range(world - 1))
    for dims, periodic in [((5, 6, 7), True), ((5, 6, 7), False)]:
        full = oracle.block_connectivity(dims, periodic)
        got = block_slab_connectivity(dims, periodic, 13, 57).numpy()
        assert np.array_equal(got, full[13:57])
        assert block_slab_connectivity(dims, periodic, 0, 0).shape == (0, 8)
    del torch


def _ann_worker(rank, world, port, name, out_dir):
    """Annihilation split by grid window: each rank's slab by the oracle, the gather by the library."""
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch
    import torch.distributed as dist

    import ann_cases
    import oracle as O
    from pypsi_b200.parallel import gather_window_slabs, window_slab

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        c = ann_cases.make(name)
        i0, i1, sub_n, sub_bounds = window_slab(c["n"], c["bounds"], world, rank)
        part = O.voxelize("restatement", sub_n, sub_bounds, c["pos"], c["conn"], mass=c["mass"],
                          periodic_box=c["periodic_box"], reftol=c["reftol"], maxlvl=c["maxlvl"],
                          mode="annihilation")["m"]
        m = torch.zeros(c["n"], dtype=torch.float64)
        gather_window_slabs(m, torch.from_numpy(part))
        np.save(os.path.join(out_dir, f"ann{rank}.npy"), m.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("block3", 2), ("block6", 3), ("window3", 2), ("tets", 3)])
def test_annihilation_window_slabs_match_single(oracle, tmp_path, name, world):
    """Open meshes (the split is for them only, see pypsi_b200.parallel)."""
    import torch.multiprocessing as mp

    import ann_cases

    mp.start_processes(_ann_worker, args=(world, _free_port(), name, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    ref = ann_cases.run_oracle(ann_cases.make(name))["m"]
    outs = [np.load(os.path.join(tmp_path, f"ann{r}.npy")) for r in range(world)]
    for r in range(1, world):
        assert np.array_equal(outs[r], outs[0])
    scale = np.abs(ref).max()
    assert scale > 0 and np.abs(outs[0] - ref).max() <= TOL * scale


def _vdf_worker(rank, world, port, out_dir):
    """Samples split by points: each rank's slab by the oracle, the gather by the library."""
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch
    import torch.distributed as dist

    import vdf_cases
    from pypsi_b200.parallel import element_slab, gather_samples

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        c = vdf_cases.make("periodic5")
        pts = np.random.default_rng(4).uniform(0, 1, (37, 3))
        p0, p1 = element_slab(len(pts), world, rank)
        res = [vdf_cases.vdf(c, "restatement", p, True) for p in pts[p0:p1]]
        counts = [len(r[0]) for r in res]
        off = torch.zeros(len(res) + 1, dtype=torch.int64)
        off[1:] = torch.cumsum(torch.tensor(counts, dtype=torch.int64), 0) if counts else off[1:]
        rho = torch.from_numpy(np.concatenate([r[0] for r in res])) if res else torch.zeros(0)
        vel = torch.from_numpy(np.concatenate([r[1] for r in res])) if res else torch.zeros((0, 3))
        o, r_, v_ = gather_samples(off, rho.to(torch.float64), vel.to(torch.float64))
        np.savez(os.path.join(out_dir, f"vdf{rank}.npz"), off=o.numpy(), rho=r_.numpy(), vel=v_.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_vdf_point_slabs_match_single(oracle, tmp_path, world):
    import torch.multiprocessing as mp

    import vdf_cases

    mp.start_processes(_vdf_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    c = vdf_cases.make("periodic5")
    pts = np.random.default_rng(4).uniform(0, 1, (37, 3))
    want = [vdf_cases.vdf(c, "restatement", p, True) for p in pts]
    for r in range(world):
        d = np.load(os.path.join(tmp_path, f"vdf{r}.npz"))
        assert d["off"][-1] == sum(len(w[0]) for w in want)
        for i, (w_rho, w_vel) in enumerate(want):
            a, b = d["off"][i], d["off"][i + 1]
            assert np.array_equal(d["rho"][a:b], w_rho) and np.array_equal(d["vel"][a:b], w_vel), (r, i)


def test_annihilation_split_refuses_periodic_meshes():
    import torch

    from pypsi_b200.parallel import annihilation_sharded

    with pytest.raises(NotImplementedError, match="open meshes only"):
        annihilation_sharded(torch.zeros((2, 2, 2), dtype=torch.float64), (2, 2, 2), ((0, 0, 0), (1, 1, 1)),
                             torch.zeros((8, 3), dtype=torch.float64), block_dims=(2, 2, 2),
                             periodic_box=((0, 0, 0), (1, 1, 1)))
