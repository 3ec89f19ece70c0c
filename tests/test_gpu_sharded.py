"""The sharded deposit on the GPU through NCCL (one rank: this run has one GPU).

voxels_sharded deposits the rank's element slab through the C ABI and runs the
exchange step as NCCL all-reduces; with one rank the slab is the whole mesh,
so the result must equal psib_voxels's to FP64 rounding (the exchange divides
and multiplies by the mass); likewise annihilation split by grid window and
phase-space samples split by points.  Several ranks are covered on the CPU by
tests/test_sharded.py.
"""
import socket
from datetime import timedelta

import numpy as np
import pytest

import cases
from pypsi_b200.metrics import field_errors

pytestmark = pytest.mark.gpu


def test_sharded_one_rank_nccl_matches(gpu):
    import torch
    import torch.distributed as dist

    from pypsi_b200 import capi
    from pypsi_b200.parallel import voxels_sharded

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        c = cases.make("c2_small")
        pos = torch.from_numpy(c["pos"].reshape(-1, 3).copy()).cuda()
        vel = torch.from_numpy(c["vel"].reshape(-1, 3).copy()).cuda()
        n = c["n"]
        shapes = {"m": n, "x": n + (3,), "v": n + (3,), "xx": n + (3, 3), "xv": n + (3, 3), "vv": n + (3, 3)}
        a = {f: torch.zeros(sh, dtype=torch.float64, device="cuda") for f, sh in shapes.items()}
        b = {f: torch.zeros(sh, dtype=torch.float64, device="cuda") for f, sh in shapes.items()}
        capi.voxels_device(a, n, c["bounds"], pos, vel, block_dims=(16, 16, 16), periodic_box=c["periodic_box"])
        voxels_sharded(b, n, c["bounds"], pos, vel, block_dims=(16, 16, 16), periodic_box=c["periodic_box"])
        torch.cuda.synchronize()
        ref = {f: t.cpu().numpy() for f, t in a.items()}
        out = {f: t.cpu().numpy() for f, t in b.items()}
        assert np.array_equal(out["m"], ref["m"])
        errs = field_errors(out, ref)
        assert max(e["norm"] for f, e in errs.items() if f != "dead_m") <= 1e-12, errs

        # annihilation split by grid window, samples split by points (one rank: the whole of each)
        import ann_cases
        import vdf_cases
        from pypsi_b200.parallel import annihilation_sharded, sample_vdf_sharded

        c = ann_cases.make("block6")
        want = ann_cases.run_oracle(c)["m"]
        m = torch.zeros(c["n"], dtype=torch.float64, device="cuda")
        annihilation_sharded(m, c["n"], c["bounds"], torch.from_numpy(c["pos"]).cuda(),
                             connectivity=torch.from_numpy(c["conn"]).cuda())
        torch.cuda.synchronize()
        assert np.abs(m.cpu().numpy() - want).max() <= 1e-12 * np.abs(want).max()
        v = vdf_cases.make("periodic5")
        pts = torch.from_numpy(np.random.default_rng(4).uniform(0, 1, (40, 3))).cuda()
        kw = dict(connectivity=torch.from_numpy(v["conn"]).cuda(), vel=torch.from_numpy(v["vel"]).cuda(),
                  mass=torch.from_numpy(v["mass"]).cuda(), periodic_box=v["periodic_box"],
                  refine_tolerance=v["reftol"], refine_max_lvl=v["maxlvl"])
        off, rho, vel = sample_vdf_sharded(pts, torch.from_numpy(v["pos"]).cuda(), **kw)
        w_off, w_rho, w_vel = capi.sample_vdf(pts, torch.from_numpy(v["pos"]).cuda(), **kw)
        assert torch.equal(off, w_off) and torch.equal(rho, w_rho) and torch.equal(vel, w_vel)
    finally:
        dist.destroy_process_group()
