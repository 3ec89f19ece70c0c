"""The capture mode (psib_options.capture): a batch deposit recorded in a CUDA graph.

A plan call (capture = 1) deposits as a plain call does and sizes every buffer;
the capture call (capture = 2) then runs with no host synchronisation and no
allocation, so torch.cuda.graph can record it.  Replays of that graph must
deposit what plain calls deposit, on the particle arrays as they are at replay
time -- the mixed atomic path on both sides, so the fields agree to rounding
(mass to 1e-12, the other fields to NORM_TOL in the voxel-scale norm) rather
than bit for bit.  The spatial tile of
the work order (psib_options.order_cell_bits) changes the order of the atomic
sums only.
"""
import numpy as np
import pytest

from pypsi_b200.metrics import field_errors
from test_gpu_batch import _cutouts

pytestmark = pytest.mark.gpu

ALL = ("m", "x", "v", "xx", "xv", "vv")


def _fields(cutouts):
    import torch

    for c in cutouts:
        c["fields"] = {f: torch.zeros(sh, dtype=torch.float64, device="cuda") for f, sh in c["shapes"].items()}
    return [{k: v for k, v in c.items() if k != "shapes"} for c in cutouts]


def _host(cutouts):
    import torch

    torch.cuda.synchronize()
    return [{f: t.cpu().numpy() for f, t in c["fields"].items()} for c in cutouts]


def _plain(cutouts, **kw):
    from pypsi_b200 import capi

    capi.voxels_batch_device(_fields(cutouts), precision="mixed", **kw)
    return _host(cutouts)


# Two orders of the same atomic sums differ by rounding; second moments of voxels made of tiny
# fragments lose digits in E[vv] - E[v]E[v] (the reference's own FP64 order and the central merge
# of the same fragments differ by ~4e-12 of a voxel's scale at these sizes), so the bound on the
# voxel-scale norm is a few times that level.
NORM_TOL = 2e-11


def _agree(a, b, what):
    for i, (s, t) in enumerate(zip(a, b)):
        assert s["m"].sum() > 0, (what, i)
        errs = field_errors(t, s)
        assert errs["m"]["rel"] <= 1e-12 and errs["dead_m"] == 0.0, (what, i, errs["m"])
        for f, e in errs.items():
            if f != "dead_m":
                assert e["norm"] <= NORM_TOL, (what, i, f, e)


def test_plan_call_deposits_as_a_plain_call(gpu):
    from pypsi_b200 import capi

    cutouts = _cutouts(16, 21, fields=ALL, lo=4, hi=10)
    want = _plain(cutouts)
    capi.voxels_batch_device(_fields(cutouts), precision="mixed", capture=1)
    _agree(want, _host(cutouts), "plan")


def test_graph_replay_equals_plain_calls(gpu):
    import torch

    from pypsi_b200 import capi
    from pypsi_b200.synth import zeldovich

    cutouts = _cutouts(16, 22, fields=ALL, lo=4, hi=10)
    want = _plain(cutouts)
    live = _fields(cutouts)
    g = capi.capture_batch(live)
    for _ in range(2):  # a replay adds to the fields as a call does
        for c in live:
            for t in c["fields"].values():
                t.zero_()
        g.replay()
        got = _host(cutouts)
        assert capi.capture_status() == 0
        _agree(want, got, "replay")

    # new particle positions in the same arrays: the graph deposits them
    for b, c in enumerate(live):
        n = c["block_dims"][0]
        side = float(c["periodic_box"][1][0])
        pos, _ = zeldovich(n, 1.2, 777 + b, box=side)
        c["pos"].copy_(torch.from_numpy(pos.reshape(-1, 3)))
        for t in c["fields"].values():
            t.zero_()
    g.replay()
    moved = _host(cutouts)
    assert capi.capture_status() == 0
    want2 = _plain(cutouts)
    _agree(want2, moved, "moved")
    del g


def test_order_cell_bits_change_only_the_order(gpu):
    cutouts = _cutouts(8, 23, fields=ALL, lo=6, hi=12)
    base = _plain(cutouts, order_cell_bits=-1)
    for bits in (3, 5, 7):
        _agree(base, _plain(cutouts, order_cell_bits=bits), bits)


def test_capture_needs_a_matching_plan(gpu):
    from pypsi_b200 import capi

    cutouts = _cutouts(3, 24, fields=("m",), lo=4, hi=5)
    capi.voxels_batch_device(_fields(cutouts), precision="mixed", capture=1)
    other = _cutouts(4, 25, fields=("m",), lo=4, hi=5)
    with pytest.raises(capi.PsibError):
        capi.voxels_batch_device(_fields(other), precision="mixed", capture=2)
    with pytest.raises(capi.PsibError):  # the capture mode is the mixed atomic deposit
        capi.voxels_batch_device(_fields(cutouts), precision="fp64", capture=1)
