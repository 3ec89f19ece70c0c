#!/usr/bin/env python
"""Throughput of PSI's phase-space-sheet voxelization on B200.

Workload: 128^3 Lagrangian particles (seeded Zel'dovich lattice, P(k) ~ k^-2,
rms displacement 2 cells, velocities 10 psi through float32) in a periodic box
of side 100, cut into 6 tets per cube and deposited with moments to order 2
(m, x, v, xx, xv, vv) on a 256^3 float64 grid.  One step = one full voxels()
call over the workload.  The headline is the mixed-precision kernel's tets/s;
the FP64 kernel is timed beside it and the mixed result is checked against it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun the ranks share out the one lattice by element slabs (strong
scaling): each deposits its slab into a full grid and one exchange combines
the grids (pypsi_b200.parallel); the step time is the max over ranks of
CUDA-event time.  `--impl reference` times the reference's own C
implementation (oracle/_ref, compiled from its sources) on all host cores over
the whole workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT]

METRIC = "tets/s @128³→256³: mixed vs FP64 GPU at ≤1e-5 voxel err; fwd+bwd / fwd time"
N_PART = 128
N_GRID = 256
RMS = 2.0
BOX = ((0.0, 0.0, 0.0), (100.0, 100.0, 100.0))
FIELDS = ["x", "v", "xx", "xv", "vv"]
WORKLOAD = "128^3 particles -> 256^3 grid, Zel'dovich rms 2 cells, fields m,x,v,xx,xv,vv"
DATA = "synthetic: seeded Zel'dovich-displaced particle lattice (P(k)~k^-2), element mass 1"
# Algorithmic bytes of one fragment: its record of 10 moments and key out of the
# walk (88 B) and the tet image's 4 positions and 4 velocities read (192 B).
ALG_BYTES_PER_FRAGMENT = 88 + 192


def clip_traffic_bytes(frags):
    """DRAM bytes the clip walk moves per step: the ncu capture of one
    64^3 -> 128^3 step (dram__bytes_read.sum + dram__bytes_write.sum over the
    walk's launches, kept with the other ncu summaries) scaled by the
    fragments of this step; None before a capture is recorded."""
    if CLIP_TRAFFIC_PER_FRAGMENT is None:
        return None
    return {"bytes_per_step": CLIP_TRAFFIC_PER_FRAGMENT * frags,
            "def": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the walk's launches in one 64^3 -> 128^3 step, "
                   f"{CLIP_TRAFFIC_PER_FRAGMENT:.0f} B per fragment, times this step's fragments"}


# bytes per fragment of the capture above (47.9 GB per call over 28.24 M fragments)
CLIP_TRAFFIC_PER_FRAGMENT = 1697.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # smaller cases for profiling runs (the headline workload is the default)
    ap.add_argument("--n-part", type=int, default=N_PART)
    ap.add_argument("--n-grid", type=int, default=N_GRID)
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the compact 512-cutout and 256^3 -> 512^3 keys")
    ap.add_argument("--ann-n", type=int, default=64, help="ann: particles per side (smaller cases for profiling)")
    ap.add_argument("--ann-grid", type=int, default=128, help="ann: grid cells per side")
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c5", "ann", "loaders", "vdf", "quad"],
                    help="c2: the headline (128^3 -> 256^3, order 2); c3: 512 uneven cutouts in one batch; "
                         "c5: 256^3 -> 512^3 with stretch refinement; ann: annihilation mode, 64^3 -> 128^3; "
                         "loaders: Gadget-2 / gevolution snapshot loading (host only); vdf: PSI.VDF at 2^20 points; "
                         "quad: 27-node elements")
    args = ap.parse_args()
    if (args.n_part, args.n_grid) != (N_PART, N_GRID) or args.precision != "both":
        args.no_cpu_baseline = True
    if (args.ann_n, args.ann_grid) != (ANN_N, ANN_GRID):
        args.no_cpu_baseline = True
    return args


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ---------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi samples taken while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if "Active" in v and "Not" not in v})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- reference arm
def arm_config(n_part=N_PART, n_grid=N_GRID, world=1):
    """The workload's config, printed identically by both arms."""
    per = ("one GPU deposits the whole lattice (seed 1234)" if world == 1 else
           f"one lattice (seed 1234) over {world} GPUs: rank r deposits element slab r into a full grid, then one "
           f"exchange (FP32 all-reduce of reference means, reduce-scatter of 34 FP64 sums per voxel over x-slabs, "
           f"all-gather)")
    return {"workload": WORKLOAD if (n_part, n_grid) == (N_PART, N_GRID) else
            f"{n_part}^3 particles -> {n_grid}^3 grid, Zel'dovich rms 2 cells, fields m,x,v,xx,xv,vv",
            "l2": "inputs larger than L2 (4.6 GB of grid fields, 3 GB of tet images per step)",
            "per_rank": per}


def slab_window(slab, nslabs, n_grid=N_GRID):
    """Voxel planes [i0, i1) of the grid along x for one of nslabs window slabs,
    and that slab's window bounds."""
    i0, i1 = n_grid * slab // nslabs, n_grid * (slab + 1) // nslabs
    d = (BOX[1][0] - BOX[0][0]) / n_grid
    return i0, i1, ((BOX[0][0] + i0 * d, BOX[0][1], BOX[0][2]), (BOX[0][0] + i1 * d, BOX[1][1], BOX[1][2]))


def _ref_inputs(seed=1234):
    """The workload's mesh as the reference takes it: positions, velocities,
    element masses and the periodic block connectivity (src/PSI.c:636-656)."""
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]
    import numpy as np

    import oracle as O
    from pypsi_b200.synth import zeldovich  # pure numpy: maps none of the library's native code

    pos, vel = zeldovich(N_PART, RMS, seed)
    conn = O.block_connectivity((N_PART,) * 3, True)
    return (np.ascontiguousarray(pos.reshape(-1, 3)), np.ascontiguousarray(vel.reshape(-1, 3)),
            np.ones(conn.shape[0]), conn)


def _ref_slab(inputs, slab, nslabs, kind, out=None, planes=None):
    """The reference's psi_voxels over the whole periodic mesh on one window slab
    of the 256^3 grid (all fields); returns (fields, seconds).  planes limits
    the slab to its first few voxel planes (the warm-up step)."""
    import oracle as O

    pos, vel, mass, conn = inputs
    i0, i1, bounds = slab_window(slab, nslabs)
    if planes is not None:
        i1 = min(i1, i0 + planes)
        d = (BOX[1][0] - BOX[0][0]) / N_GRID
        bounds = (bounds[0], (BOX[0][0] + i1 * d, bounds[1][1], bounds[1][2]))
    n = (i1 - i0, N_GRID, N_GRID)
    if out is None or out["m"].shape != n:
        out = O.new_fields(n, FIELDS)
    t0 = time.perf_counter()
    O.voxelize(kind, n=n, bounds=bounds, pos=pos, vel=vel, mass=mass, conn=conn, periodic_box=BOX, out=out)
    return out, time.perf_counter() - t0


def _ref_worker(pipe, slab, nslabs, kind):
    """One process of the reference arm: deposits its window slab of the whole
    workload at every 'step', a few voxel planes of it at every 'warm'."""
    inputs = _ref_inputs()
    out, thin = None, None
    pipe.send("ready")
    while True:
        cmd = pipe.recv()
        if cmd == "stop":
            break
        if cmd == "warm":
            thin, secs = _ref_slab(inputs, slab, nslabs, kind, thin, planes=1)
        else:
            out, secs = _ref_slab(inputs, slab, nslabs, kind, out)
        pipe.send(secs)


def run_reference(args):
    """The reference's own C path (oracle/_ref, compiled from its sources) on
    every host core over the whole workload: the 256^3 grid split along x into
    one window slab per core, each process running psi_voxels over every element
    of the periodic 128^3 mesh on its slab (periodic images and window clips
    are the reference's own).  The slabs are disjoint, so together they are the
    full deposit (to rounding at the slab faces).  A step is the wall time from
    the start of all slabs to the end of the last."""
    rank, world, _ = env_rank()
    if rank != 0:
        return
    import multiprocessing as mp

    sys.path[:0] = [os.path.join(ROOT, "oracle")]
    import oracle as O

    kind = "reference" if O.available("reference") else "restatement"
    cores = len(os.sched_getaffinity(0))
    ctx = mp.get_context("spawn")
    pipes, procs = [], []
    for slab in range(cores):
        a, b = ctx.Pipe()
        p = ctx.Process(target=_ref_worker, args=(b, slab, cores, kind), daemon=True)
        p.start()
        pipes.append(a)
        procs.append(p)
    try:
        for a in pipes:
            assert a.recv() == "ready"

        def step(cmd):
            t0 = time.perf_counter()
            for a in pipes:
                a.send(cmd)
            inner = max(a.recv() for a in pipes)
            return time.perf_counter() - t0, inner

        for _ in range(args.warmup):
            step("warm")
        times = [step("step") for _ in range(args.steps)]
    finally:
        for a in pipes:
            try:
                a.send("stop")
            except OSError:
                pass
        for p in procs:
            p.join(30)
    secs = sum(t[0] for t in times)
    tets = 6 * N_PART ** 3 * args.steps
    value = tets / secs
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "tets/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
            "config": arm_config(world=world),
            "precision": "fp64 (the reference's own C code)",
            "cpu_baseline": {"value": value, "unit": "tets/s", "cores": cores,
                             "kind": "reference" if kind == "reference" else "port",
                             "sample": f"the whole workload every step: the 256^3 grid in {cores} window slabs "
                                       f"along x, one process per slab, each running psi_voxels over all "
                                       f"{N_PART ** 3} elements of the periodic mesh (periodic images included)"},
            "warmup_step": "each process deposits the first voxel plane of its slab",
            "slowest_slab_ms_per_step": 1000 * sum(t[1] for t in times) / args.steps,
            "e2e": {"value": value, "unit": "tets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_single(nslabs=16, slab=0):
    """The reference's C path on one host core over a bounded sample: one of
    nslabs window slabs of the whole workload (slab 0 holds the periodic wrap
    at x = 0), every element of the mesh given.  Returns the baseline line and
    the reference's fields on that slab (the parity sample of the GPU arm)."""
    sys.path[:0] = [os.path.join(ROOT, "oracle")]
    import oracle as O

    kind = "reference" if O.available("reference") else "restatement"
    inputs = _ref_inputs()
    out, secs = _ref_slab(inputs, slab, nslabs, kind)
    tets = 6 * N_PART ** 3 / nslabs
    return {"value": tets / secs, "unit": "tets/s", "cores": 1, "kind": "reference" if kind == "reference" else "port",
            "sample": f"window slab {slab} of {nslabs} along x of the 256^3 grid (1/{nslabs} of the workload, "
                      f"{secs:.1f} s), psi_voxels over all {N_PART ** 3} elements of the periodic mesh; tets counted "
                      f"as 6 n^3 / {nslabs}"}, out


def parity_on_slab(ref, deposit, nslabs=16, slab=0):
    """The GPU's FP64 and mixed fields on the CPU-baseline sample's window
    against the reference's: FP64 bit for bit; mixed within 1e-5 of the
    reference plus the reference's own rounding (its distance to the
    FP64-central result), per field in the voxel-scale normalisation."""
    import numpy as np

    from pypsi_b200.metrics import error_maps, field_errors

    i0, i1, bounds = slab_window(slab, nslabs)
    n = (i1 - i0, N_GRID, N_GRID)
    outs = {p: deposit(n, bounds, p) for p in ("fp64", "mixed", "fp64-central")}
    e_mr = error_maps(outs["mixed"], ref, scale_from=outs["fp64-central"])
    e_rc = error_maps(ref, outs["fp64-central"])
    return {"sample": f"window slab {slab} of {nslabs} along x (the CPU-baseline sample), all fields, against the "
                      f"reference's own C code",
            "fp64_bitwise": all(bool(np.array_equal(outs["fp64"][f], ref[f])) for f in ref),
            "mixed_err_vs_reference": {f: e["norm"] for f, e in field_errors(outs["mixed"], ref).items()
                                       if f != "dead_m"},
            "mixed_within_1e5_plus_reference_rounding": all(bool(np.all(e_mr[f] <= 1e-5 + e_rc[f])) for f in e_mr)}


# ---------------------------------------------------------------- annihilation (--workload ann)
ANN_N, ANN_GRID, ANN_RMS = 64, 128, 1.5
ANN_METRIC = "tet pairs/s @64³→128³ annihilation (m += rho0 rho1 V over overlapping tets), FP64"
ANN_WORKLOAD = ("64^3 particles, open lattice (63^3 trilinear elements), Zel'dovich rms 1.5 cells -> 128^3 grid "
                "over the box, annihilation mode, m only")
ANN_DATA = "synthetic: seeded Zel'dovich-displaced particle lattice (P(k)~k^-2), unwrapped, element mass 1"


def _ann_init(seed):
    global _A
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]
    from pypsi_b200.synth import zeldovich

    _A = zeldovich(ANN_N, ANN_RMS, seed, wrap=False)[0]


def ann_blocks(edge=16):
    nb = (ANN_N - 1) // edge
    return [(i * edge, j * edge, k * edge) for i in range(nb) for j in range(nb) for k in range(nb)]


def _ann_block(args):
    """Annihilation of the elements of one Lagrangian sub-block (edge^3 elements)
    on a window covering it at the workload's voxel size: the reference's
    psi_voxels times it; the oracle's restatement (not timed) counts its tet
    pairs.  Returns (tet pairs, seconds)."""
    origin, edge, kind = args
    import numpy as np

    import oracle as O

    i0, j0, k0 = origin
    p = np.ascontiguousarray(_A[i0:i0 + edge + 1, j0:j0 + edge + 1, k0:k0 + edge + 1].reshape(-1, 3))
    conn = O.block_connectivity((edge + 1,) * 3, False)
    d = BOX[1][0] / ANN_GRID
    lo = np.floor(p.min(axis=0) / d) - 1
    hi = np.ceil(p.max(axis=0) / d) + 1
    bounds = (tuple(lo * d), tuple(hi * d))
    ng = tuple(int(v) for v in (hi - lo))
    t0 = time.perf_counter()
    O.voxelize(kind, n=ng, bounds=bounds, pos=p, conn=conn, mode="annihilation")
    secs = time.perf_counter() - t0
    _, cnt = O.voxelize("restatement", n=ng, bounds=bounds, pos=p, conn=conn, mode="annihilation", counters=True)
    return cnt["tet_images"], secs


def _ann_sample_line(kind, nb, pairs, secs, cores, per="per step"):
    return {"value": pairs / secs, "unit": "tet pairs/s", "cores": cores,
            "kind": "reference" if kind == "reference" else "port",
            "sample": f"{nb} Lagrangian 16^3-element sub-blocks of the workload {per} ({pairs} tet pairs, "
                      f"{secs:.1f} s of the reference's psi_voxels), each on a window covering it at the 128^3 "
                      f"voxel size; tet pairs counted by the oracle"}


def run_reference_ann(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return
    import multiprocessing as mp

    sys.path[:0] = [os.path.join(ROOT, "oracle")]
    import oracle as O

    kind = "reference" if O.available("reference") else "restatement"
    cores = len(os.sched_getaffinity(0))
    blocks = ann_blocks()
    per_step = blocks[: max(1, min(len(blocks), cores))]
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_ann_init, initargs=(4242,)) as pool:
        def step():
            t0 = time.perf_counter()
            res = pool.map(_ann_block, [(b, 16, kind) for b in per_step], chunksize=1)
            return sum(r[0] for r in res), time.perf_counter() - t0

        for _ in range(args.warmup):
            step()
        pairs, secs = 0, 0.0
        for _ in range(args.steps):
            t, s_ = step()
            pairs += t
            secs += s_
    value = pairs / secs
    line = {"impl": "reference", "metric": ANN_METRIC, "value": value, "unit": "tet pairs/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": ANN_DATA,
            "config": {"workload": ANN_WORKLOAD, "precision": "fp64 (reference C)"},
            "cpu_baseline": _ann_sample_line(kind, len(per_step), pairs, secs, cores, "per step, one per process"),
            "e2e": {"value": value, "unit": "tet pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    line["cpu_baseline"]["value"] = value
    print(json.dumps(line), flush=True)


def run_ann(args):
    """Annihilation of a 64^3 open lattice on a 128^3 grid: device-resident
    timing through the C ABI, and the drop-in module on host arrays (e2e)."""
    import numpy as np
    import torch

    from pypsi_b200 import PSI, capi
    from pypsi_b200.synth import zeldovich

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n_part, n_grid = args.ann_n, args.ann_grid
    pos = zeldovich(n_part, ANN_RMS, 4242 + rank, wrap=False)[0]
    dpos = torch.from_numpy(pos.reshape(-1, 3)).to(dev)
    m = torch.zeros((n_grid,) * 3, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()

    def step():
        return capi.voxels_device({"m": m}, (n_grid,) * 3, BOX, dpos, block_dims=(n_part,) * 3, mode="annihilation",
                                  stream=stream)

    for _ in range(max(1, args.warmup)):
        m.zero_()
        st = step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ck = Clocks(local)
    ck.__enter__()
    e0.record(stream)
    stats = [step() for _ in range(args.steps)]
    e1.record(stream)
    torch.cuda.synchronize()
    ck.__exit__()
    ms = e0.elapsed_time(e1) / args.steps
    pairs = st["tet_images"]
    # end to end: PSI.voxels(mode='annihilation') on host arrays (the copies in the timed region)
    e2e = None
    if not args.no_e2e:
        grid = PSI.Grid(n=(n_grid,) * 3, bounds=BOX)
        mesh = PSI.Mesh(loader="block", pos=np.ascontiguousarray(pos))
        PSI.voxels(grid=grid, mesh=mesh, mode="annihilation")
        ts = []
        for _ in range(max(1, args.e2e_steps)):
            grid.fields["m"][...] = 0.0
            t0 = time.perf_counter()
            PSI.voxels(grid=grid, mesh=mesh, mode="annihilation")
            ts.append(time.perf_counter() - t0)
        t = statistics.median(ts)
        e2e = {"value": pairs / t, "unit": "tet pairs/s", "h2d_bytes_per_step": int(pos.nbytes + grid.fields["m"].nbytes),
               "d2h_bytes_per_step": int(grid.fields["m"].nbytes), "api": "PSI.voxels(grid, mesh, mode='annihilation')"
               " on host numpy arrays", "ms_per_step": 1000 * t}
    line = {"metric": ANN_METRIC, "value": pairs / (ms * 1e-3), "unit": "tet pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": ANN_DATA,
            "config": {"workload": ANN_WORKLOAD if (n_part, n_grid) == (ANN_N, ANN_GRID) else
                       f"{n_part}^3 particles, open lattice, Zel'dovich rms 1.5 cells -> {n_grid}^3 grid, annihilation",
                       "l2": "inputs larger than L2 (tet records and fragment records)"},
            "work": {"elements_kept": st["elements_kept"], "tets": st["tets"], "tet_pairs": pairs,
                     "fragments": st["fragments"], "splits": st["splits"], "chunks": st["chunks"]},
            "stage_ms": {"elements_pairs_and_tet_pairs": st["ms_tess"], "clip": st["ms_clip"],
                         "sort_and_apply": st["ms_final"]},
            "gpu_launches": int(sum(x["kernel_launches"] for x in stats)), "clocks": ck.summary()}
    if e2e:
        line["e2e"] = e2e
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path[:0] = [os.path.join(ROOT, "oracle")]
        import oracle as O

        kind = "reference" if O.available("reference") else "restatement"
        _ann_init(4242)
        pairs_c, secs, nb = 0, 0.0, 0
        for b in ann_blocks():
            pc, sc = _ann_block((b, 16, kind))
            pairs_c += pc
            secs += sc
            nb += 1
            if secs > 12.0:
                break
        line["cpu_baseline"] = _ann_sample_line(kind, nb, pairs_c, secs, 1, "in all")
    capi.lib.psib_release_device_memory()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- PSI.VDF (--workload vdf)
VDF_N, VDF_POINTS = 64, 1 << 20
VDF_METRIC = "sample points/s, PSI.VDF batched at 2^20 random points of a 64³ periodic sheet (rms 2 cells)"


def run_vdf(args):
    """Phase-space samples at 2^20 random points of a periodic 64^3 Zel'dovich
    sheet (rms 2 cells, box 100, the tree's window = the box), unrefined:
    psib_sample_vdf on device arrays (CUDA events), the same on host arrays
    (e2e), and the reference's psi_sample_vdf per point over its own tree."""
    import numpy as np
    import torch

    from pypsi_b200 import capi
    from pypsi_b200.synth import zeldovich

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pos, vel = zeldovich(VDF_N, 2.0, 777 + rank)
    pts = np.random.default_rng(5 + rank).uniform(0.0, 100.0, (VDF_POINTS, 3))
    dpos = torch.from_numpy(pos.reshape(-1, 3)).to(dev)
    dvel = torch.from_numpy(vel.reshape(-1, 3)).to(dev)
    dpts = torch.from_numpy(pts).to(dev)
    kw = dict(block_dims=(VDF_N,) * 3, periodic_box=BOX)

    def step():
        return capi.sample_vdf(dpts, dpos, vel=dvel, **kw)

    for _ in range(max(1, args.warmup)):
        off, rho, v = step()
    torch.cuda.synchronize()
    nsamp = int(off[-1].item())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ck = Clocks(local)
    ck.__enter__()
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ck.__exit__()
    ms = e0.elapsed_time(e1) / args.steps
    line = {"metric": VDF_METRIC, "value": VDF_POINTS / (ms * 1e-3), "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
            "config": {"workload": "64^3 periodic lattice (box 100, rms 2 cells), 2^20 uniform points, no refinement, "
                                   "tree window = the box", "samples": nsamp},
            "gpu_launches": None, "clocks": ck.summary()}
    if not args.no_e2e:
        capi.sample_vdf(pts, pos.reshape(-1, 3), vel=vel.reshape(-1, 3), **kw)
        ts = []
        for _ in range(max(1, args.e2e_steps)):
            t0 = time.perf_counter()
            capi.sample_vdf(pts, pos.reshape(-1, 3), vel=vel.reshape(-1, 3), **kw)
            ts.append(time.perf_counter() - t0)
        t = statistics.median(ts)
        line["e2e"] = {"value": VDF_POINTS / t, "unit": "points/s", "h2d_bytes_per_step": int(pts.nbytes + pos.nbytes +
                       vel.nbytes), "d2h_bytes_per_step": int(8 * (VDF_POINTS + 1) + 32 * nsamp),
                       "api": "capi.sample_vdf on host numpy arrays (psib_sample_vdf, host memory)",
                       "ms_per_step": 1000 * t}
    if not args.no_e2e:
        # the drop-in call one point at a time, as a loop over the reference's PSI.VDF with a tree would run
        from pypsi_b200 import PSI

        mesh = PSI.Mesh(loader="block", pos=pos, vel=vel, periodic_box=BOX)
        tree = PSI.RStarTree(mesh)
        PSI.VDF(mesh, tuple(pts[0]), tree)
        npt = 2000
        t0 = time.perf_counter()
        for p in pts[:npt]:
            PSI.VDF(mesh, tuple(p), tree)
        t = time.perf_counter() - t0
        line["one_point_per_call"] = {"value": npt / t, "unit": "points/s",
                                      "api": "PSI.VDF(mesh, point, tree) in a Python loop, the tree's device index "
                                             "built by the first call"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path[:0] = [os.path.join(ROOT, "oracle")]
        import oracle as O

        kind = "reference" if O.available("reference") else "restatement"
        conn = O.block_connectivity((VDF_N,) * 3, True)
        n = 1 << 18 if kind == "reference" else 64  # the reference: ~47 K points/s after a ~4 s tree build
        _, secs = O.sample_vdf_many(kind, pos.reshape(-1, 3), conn, pts[:n], vel=vel.reshape(-1, 3),
                                    periodic_box=BOX, window=BOX)
        line["cpu_baseline"] = {"value": n / secs, "unit": "points/s", "cores": 1,
                                "kind": "reference" if kind == "reference" else "port",
                                "sample": f"the first {n} points, psi_sample_vdf per point over a tree built once "
                                          f"({secs:.1f} s)"}
    capi.lib.psib_release_device_memory()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- triquadratic elements (--workload quad)
def quad_mesh(ne, seed, box=100.0):
    """27-node elements: node (a,b,c) of element (i,j,k) is point (2i+a, 2j+b, 2k+c) of an open
    (2 ne + 1)^3 lattice of the box, displaced by a Zel'dovich field (rms 1 lattice cell)."""
    import numpy as np

    from pypsi_b200.synth import zeldovich

    nn = 2 * ne + 1
    pos, vel = zeldovich(nn, 1.0, seed, box=box * nn / (nn - 1), wrap=False)
    conn = np.empty((ne, ne, ne, 27), dtype=np.int32)
    i, j, k = np.meshgrid(np.arange(ne), np.arange(ne), np.arange(ne), indexing="ij")
    for a in range(3):
        for b in range(3):
            for c in range(3):
                conn[..., 9 * a + 3 * b + c] = ((2 * i + a) * nn + (2 * j + b)) * nn + (2 * k + c)
    return pos.reshape(-1, 3), vel.reshape(-1, 3), conn.reshape(-1, 27)


def run_quad(args):
    """32^3 triquadratic elements (65^3 nodes) on 128^3 voxels, all order-2
    fields, unrefined: mixed and FP64 tets/s on device arrays, the reference's
    psi_voxels on 4^3-element sub-blocks (own window at the same voxel size)."""
    import numpy as np
    import torch

    from pypsi_b200 import capi

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ne, ng = 32, 128
    pos, vel, conn = quad_mesh(ne, 31 + rank)
    dpos, dvel = torch.from_numpy(pos).to(dev), torch.from_numpy(vel).to(dev)
    dconn = torch.from_numpy(conn).to(dev)
    shapes = {"m": (), "x": (3,), "v": (3,), "xx": (3, 3), "xv": (3, 3), "vv": (3, 3)}
    fields = {f: torch.zeros((ng,) * 3 + sh, dtype=torch.float64, device=dev) for f, sh in shapes.items()}
    out = {}
    for prec in ("mixed", "fp64"):
        def step():
            return capi.voxels_device(fields, (ng,) * 3, BOX, dpos, dvel, connectivity=dconn, precision=prec)

        for _ in range(max(1, args.warmup)):
            st = step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        out[prec] = (e0.elapsed_time(e1) / args.steps, st)
    ms, st = out["mixed"]
    line = {"metric": "tets/s, 27-node elements 32³ (65³ nodes) → 128³, order 2, mixed", "value": st["tets"] / (ms * 1e-3),
            "unit": "tets/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic: seeded Zel'dovich-displaced open node lattice, element mass 1",
            "config": {"workload": "32^3 triquadratic elements on a 128^3 grid over the box, fields m,x,v,xx,xv,vv, "
                                   "no refinement"},
            "fp64": {"value": out["fp64"][1]["tets"] / (out["fp64"][0] * 1e-3), "ms_per_step": out["fp64"][0]},
            "work": {"tets": st["tets"], "fragments": st["fragments"]}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path[:0] = [os.path.join(ROOT, "oracle")]
        import oracle as O

        if O.available("reference"):
            d = BOX[1][0] / ng
            tets, secs, nb = 0, 0.0, 0
            c4 = conn.reshape(ne, ne, ne, 27)
            for o in range(0, ne ** 3 // 64):
                a, b, c = 4 * (o // 64), 4 * ((o // 8) % 8), 4 * (o % 8)
                sub = np.ascontiguousarray(c4[a:a + 4, b:b + 4, c:c + 4].reshape(-1, 27))
                p = pos[np.unique(sub)]
                lo, hi = np.floor(p.min(0) / d) - 1, np.ceil(p.max(0) / d) + 1
                t0 = time.perf_counter()
                O.voxelize("reference", n=tuple(int(v) for v in hi - lo), bounds=(tuple(lo * d), tuple(hi * d)),
                           pos=pos, vel=vel, conn=sub, fields=FIELDS)
                secs += time.perf_counter() - t0
                tets += 6 * sub.shape[0]
                nb += 1
                if secs > 10.0:
                    break
            line["cpu_baseline"] = {"value": tets / secs, "unit": "tets/s", "cores": 1, "kind": "reference",
                                    "sample": f"{nb} sub-blocks of 4^3 elements ({tets} tets, {secs:.1f} s), each on "
                                              "a window covering it at the 128^3 voxel size"}
    capi.lib.psib_release_device_memory()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- snapshot loaders (--workload loaders)
def run_loaders(args):
    """Host code only: PSI.Mesh(loader='gadget2' | 'gevolution') on a synthetic
    128^3 snapshot (a seeded displaced lattice in shuffled file order, read from
    the page cache) against the reference's own load_gadget2 / load_gevolution
    (oracle/_ref), in particles/s; every array is compared."""
    import numpy as np

    sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]
    import oracle as O
    from snapshots import make_snapshot

    from pypsi_b200 import PSI

    rank, _, _ = env_rank()
    if rank != 0:
        return
    n = 128
    lines = []
    with tempfile.TemporaryDirectory() as d:
        for flav in ("gadget2", "gevolution"):
            path = os.path.join(d, flav)
            make_snapshot(path, n, flavour=flav, seed=1)
            open(path, "rb").read()
            ours, ref = [], []
            for _ in range(max(1, args.warmup)):
                mesh = PSI.Mesh(loader=flav, filename=path)
            for _ in range(args.steps):
                t0 = time.perf_counter()
                mesh = PSI.Mesh(loader=flav, filename=path)
                ours.append(time.perf_counter() - t0)
                if O.available("reference"):
                    t0 = time.perf_counter()
                    r = O.load_snapshot("reference", path, flav)
                    ref.append(time.perf_counter() - t0)
            same = None
            if ref:
                same = all(np.array_equal(a, b) for a, b in zip((mesh.pos, mesh.vel, mesh.mass, mesh.connectivity),
                                                                 r[:4]))
            t = statistics.median(ours)
            line = {"metric": f"particles/s loaded, {flav} snapshot of 128^3 particles", "value": n ** 3 / t,
                    "unit": "particles/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
                    "ms_per_step": 1000 * t, "higher_is_better": True, "scaling": "none", "vs_baseline": None,
                    "dtype": "f32->f64", "data": "synthetic: seeded displaced lattice, shuffled file order",
                    "config": {"workload": f"PSI.Mesh(loader='{flav}') of a {os.path.getsize(path) >> 20} MiB file "
                                           "in the page cache, host threads " + str(len(os.sched_getaffinity(0)))},
                    "arrays_equal_reference": same}
            if ref:
                tr = statistics.median(ref)
                line["cpu_baseline"] = {"value": n ** 3 / tr, "unit": "particles/s", "cores": 1, "kind": "reference",
                                        "sample": "the same file through the reference's own loader"}
            lines.append(line)
    for line in lines:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
def time_fwd_bwd(x0, n_part, n_grid, steps, warmup, barrier):
    """CUDA-event time of the forward pass of a density loss and of forward +
    backward, on particles x0 ((n_part^3, 3) float64 on the GPU)."""
    import torch

    from pypsi_b200.autograd import deposit_density

    dv = (BOX[1][0] - BOX[0][0]) ** 3 / n_grid ** 3
    kw = dict(n=(n_grid,) * 3, bounds=BOX, block_dims=(n_part,) * 3, periodic_box=BOX)
    g = torch.Generator(device=x0.device).manual_seed(7)
    cell = (BOX[1][0] - BOX[0][0]) / n_part
    with torch.no_grad():
        rho_t = deposit_density(x0 + 0.05 * cell * torch.randn(x0.shape, generator=g, device=x0.device,
                                                                dtype=torch.float64), **kw) / dv
    x = x0.clone().requires_grad_(True)

    def fwd():
        with torch.no_grad():
            return ((deposit_density(x, **kw) / dv - rho_t) ** 2).sum()

    def fwd_bwd():
        x.grad = None
        loss = ((deposit_density(x, **kw) / dv - rho_t) ** 2).sum()
        loss.backward()
        return loss

    out = {}
    stream = torch.cuda.current_stream()
    for name, fn in (("fwd", fwd), ("fwd_bwd", fwd_bwd)):
        for _ in range(warmup):
            fn()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        out[name + "_ms"] = e0.elapsed_time(e1) / steps
    out["ratio"] = out["fwd_bwd_ms"] / out["fwd_ms"]
    out["tets_per_s_fwd_bwd"] = 6 * n_part ** 3 / (out["fwd_bwd_ms"] * 1e-3)
    return out


def run_c3(args):
    print(json.dumps(c3_result(args, args.steps, args.warmup)), flush=True)


def c3_result(args, steps, warmup):
    """512 independent cutouts, edge n log-uniform in [8, 64], Zel'dovich rms 1.5
    cells in their own periodic box of side 100, density on their own (2n)^3 grid:
    one psib_voxels_batch call against 512 separate psib_voxels calls."""
    import math

    import numpy as np
    import torch

    from pypsi_b200 import capi
    from pypsi_b200.synth import zeldovich

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    rng = np.random.default_rng(333 + rank)
    ns = [int(round(math.exp(rng.uniform(math.log(8), math.log(64))))) for _ in range(512)]
    cut = []
    for b, n in enumerate(ns):
        pos, _ = zeldovich(n, 1.5, 10000 + 512 * rank + b)
        cut.append(dict(n=(2 * n,) * 3, bounds=BOX, pos=torch.from_numpy(pos.reshape(-1, 3)).cuda(),
                        block_dims=(n,) * 3, periodic_box=BOX,
                        fields={"m": torch.zeros((2 * n,) * 3, dtype=torch.float64, device="cuda")}))
    tets = sum(6 * n ** 3 for n in ns)
    stream = torch.cuda.current_stream()

    # the queue capacity and work-order tile of this batch, picked by timing (the batch is
    # deposited many times)
    tune = capi.autotune_batch(cut, precision="mixed", repeats=1)
    kw = {"queue_voxels": tune["queue_voxels"], "order_cell_bits": tune["order_cell_bits"]}

    def batch():
        return capi.voxels_batch_device(cut, precision="mixed", stream=stream, **kw)

    def separate():
        return [capi.voxels_device(c["fields"], c["n"], c["bounds"], c["pos"], block_dims=c["block_dims"],
                                   periodic_box=c["periodic_box"], precision="mixed", stream=stream) for c in cut]

    def timed(fn, steps):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = [fn() for _ in range(steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, out

    ck = Clocks(local)
    ck.__enter__()
    ms_b, st_b = timed(batch, steps)
    ck.__exit__()
    ms_s, _ = timed(separate, max(1, steps // 2))
    # the same batch recorded once as a CUDA graph (capture mode: no host synchronisation), replayed
    try:
        graph = capi.capture_batch(cut, precision="mixed", **kw)
        ms_g, _ = timed(graph.replay, steps)
        graph_line = {"value": tets / (ms_g * 1e-3), "ms_per_step": ms_g, "status": capi.capture_status()}
        del graph
    except capi.PsibError as e:
        graph_line = {"unavailable": str(e)}
    line = {"metric": "tets/s, 512 uneven cutouts (n in [8,64], (2n)^3 grids, density), one batch call", "value":
            tets / (ms_b * 1e-3), "unit": "tets/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
            "ms_per_step": ms_b, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic: 512 seeded Zel'dovich lattices, rms 1.5 cells, element mass 1",
            "config": {"workload": "512 cutouts, edge log-uniform in [8,64], own box of side 100, (2n)^3 grids, m only",
                       "precision": "mixed"},
            "separate_calls": {"value": tets / (ms_s * 1e-3), "ms_per_step": ms_s, "calls": 512},
            "batch_over_separate": ms_s / ms_b,
            "graph_replay": graph_line,
            "autotuned": {"queue_voxels": kw["queue_voxels"], "order_cell_bits": kw["order_cell_bits"]}, "work": {"tets": tets, "cutouts": 512, "edge_min": min(ns),
                                                         "edge_max": max(ns)},
            "gpu_launches": int(st_b[-1]["kernel_launches"]), "clocks": ck.summary()}
    capi.lib.psib_release_device_memory()
    return line


def run_c5(args):
    print(json.dumps(c5_result(args, args.steps, args.warmup)), flush=True)


def c5_result(args, steps, warmup):
    """256^3 particles (rms 3 cells) onto 512^3, fields m and v, mixed precision,
    tets refined up to 2 levels where a (sub)cube's volume or edge stretches
    beyond 8x its Lagrangian value; total mass must be 256^3 to 1e-13."""
    import torch

    from pypsi_b200 import capi
    from pypsi_b200.metrics import mass_error
    from pypsi_b200.synth import zeldovich

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    n_part, n_grid = 256, 512
    pos, vel = zeldovich(n_part, 3.0, 5555 + rank)
    dev = torch.device("cuda", local)
    dpos = torch.from_numpy(pos.reshape(-1, 3)).to(dev)
    dvel = torch.from_numpy(vel.reshape(-1, 3)).to(dev)
    del pos, vel
    fields = {"m": torch.zeros((n_grid,) * 3, dtype=torch.float64, device=dev),
              "v": torch.zeros((n_grid,) * 3 + (3,), dtype=torch.float64, device=dev)}
    stream = torch.cuda.current_stream()

    def step():
        return capi.voxels_device(fields, (n_grid,) * 3, BOX, dpos, dvel, block_dims=(n_part,) * 3,
                                  periodic_box=BOX, precision="mixed", refine_tolerance=8.0, refine_max_lvl=2,
                                  refine_criterion="stretch", stream=stream)

    for f in fields.values():
        f.zero_()
    st = step()
    torch.cuda.synchronize()
    merr = mass_error(fields["m"].cpu().numpy(), n_part ** 3)
    for _ in range(max(0, warmup - 1)):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ck = Clocks(local)
    ck.__enter__()
    e0.record(stream)
    stats = [step() for _ in range(steps)]
    e1.record(stream)
    torch.cuda.synchronize()
    ck.__exit__()
    ms = e0.elapsed_time(e1) / steps
    tets = st["tets"]
    line = {"metric": "tets/s @256³→512³ (stretch refinement 8x, 2 levels), mixed, fields m,v", "value": tets / (ms * 1e-3),
            "unit": "tets/s", "n_gpus": 1, "steps": steps, "warmup": warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic: seeded Zel'dovich lattice 256^3, rms 3 cells, element mass 1",
            "config": {"workload": "256^3 particles -> 512^3 grid, fields m,v, stretch refinement 8x up to 2 levels",
                       "l2": "inputs larger than L2"},
            "work": {"tets_after_refinement": tets, "unrefined_tets": 6 * n_part ** 3, "tet_images": st["tet_images"],
                     "fragments": st["fragments"], "chunks": st["chunks"]},
            "mass_err_mixed": merr, "stage_ms": {"tessellate_and_order": st["ms_tess"], "clip": st["ms_clip"],
                                                 "sort_and_apply": st["ms_final"]},
            "gpu_launches": int(sum(x["kernel_launches"] for x in stats)), "clocks": ck.summary()}
    del fields
    capi.lib.psib_release_device_memory()
    return line


def run_ours(args):
    import numpy as np
    import torch

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    from pypsi_b200 import PSI, capi
    from pypsi_b200.metrics import error_maps, field_errors, mass_error
    from pypsi_b200.synth import zeldovich

    n_part, n_grid = args.n_part, args.n_grid
    # one GPU: the whole mesh.  Several: one mesh shared out by element slabs (strong scaling),
    # every rank depositing its slab and one exchange combining the grids
    sharded = world > 1
    tets_per_step = 6 * n_part ** 3
    fp64_peak = capi.measure_fma_peak("fp64")
    fp32_peak = capi.measure_fma_peak("fp32")
    pos, vel = zeldovich(n_part, RMS, 1234)
    dev = torch.device("cuda", local)
    dpos = torch.from_numpy(pos.reshape(-1, 3)).to(dev)
    dvel = torch.from_numpy(vel.reshape(-1, 3)).to(dev)
    shapes = {"m": (n_grid,) * 3, "x": (n_grid,) * 3 + (3,), "v": (n_grid,) * 3 + (3,)}
    for f in ("xx", "xv", "vv"):
        shapes[f] = (n_grid,) * 3 + (3, 3)

    def fresh():
        return {f: torch.zeros(s, dtype=torch.float64, device=dev) for f, s in shapes.items()}

    stream = torch.cuda.current_stream()
    if sharded:
        from pypsi_b200.parallel import block_slab_connectivity, element_slab, merge_fields

        e0, e1 = element_slab(n_part ** 3, world, rank)
        slab_conn = block_slab_connectivity((n_part,) * 3, True, e0, e1, device=dev)

    def step(fields, prec, n=(n_grid,) * 3, bounds=BOX):
        if not sharded:
            return capi.voxels_device(fields, n, bounds, dpos, dvel, block_dims=(n_part,) * 3,
                                      periodic_box=BOX, precision=prec, stream=stream)
        # voxels_sharded's steps, keeping the library's stats of this rank's slab
        for t in fields.values():
            t.zero_()
        st = capi.voxels_device(fields, n, bounds, dpos, dvel, connectivity=slab_conn, periodic_box=BOX,
                                precision=prec, stream=stream)
        merge_fields(fields)
        return st

    def barrier():
        if dist:
            dist.barrier()

    def timed(prec, fields, clocks=False):
        for _ in range(args.warmup):
            step(fields, prec)
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stats = []
        ck = Clocks(local) if clocks else None
        if ck:
            ck.__enter__()
        e0.record(stream)
        for _ in range(args.steps):
            stats.append(step(fields, prec))
        e1.record(stream)
        torch.cuda.synchronize()
        if ck:
            ck.__exit__()
        barrier()
        ms = e0.elapsed_time(e1)
        if dist:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms / args.steps, stats, (ck.summary() if ck else None)

    fields = fresh()
    head = "fp64" if args.precision == "fp64" else "mixed"
    ms_mixed, st_mixed, clocks = timed(head, fields, clocks=True)
    ms_fp64, st_fp64 = ms_mixed, st_mixed
    if args.precision == "both":
        ms_fp64, st_fp64, _ = timed("fp64", fields)
    del fields

    # accuracy of the headline (mixed) against FP64 on the same input, and mass.
    # FP64-central (the FP64 walk with per-fragment central moments) stands in
    # for the exact result: the reference-order FP64 result carries its own
    # rounding in voxels of tiny fragments.
    errs, errs_x, errs_rx, merr, within = {}, {}, {}, {}, None
    if args.precision == "both" and not sharded:
        outs = {}
        for prec in ("fp64", "mixed", "fp64-central"):
            f = fresh()
            step(f, prec)
            torch.cuda.synchronize()
            outs[prec] = {k: v.cpu().numpy() for k, v in f.items()}
            merr[prec] = mass_error(outs[prec]["m"], n_part ** 3)
            del f
        errs = field_errors(outs["mixed"], outs["fp64"])
        errs_x = field_errors(outs["mixed"], outs["fp64-central"])
        errs_rx = field_errors(outs["fp64"], outs["fp64-central"])
        e_or = error_maps(outs["mixed"], outs["fp64"], scale_from=outs["fp64-central"])
        e_rx = error_maps(outs["fp64"], outs["fp64-central"])
        within = all(bool(np.all(e_or[f] <= 1e-5 + e_rx[f])) for f in e_or)
        del outs, e_or, e_rx
    torch.cuda.empty_cache()

    # end to end through the drop-in module: host numpy in, host numpy out
    e2e = None
    if not args.no_e2e and sharded:
        # several GPUs: parallel.voxels_sharded, every step copying the mesh in from pinned host
        # memory and rank 0 copying the merged fields back
        from pypsi_b200.parallel import voxels_sharded

        hpos = torch.from_numpy(pos.reshape(-1, 3)).pin_memory()
        hvel = torch.from_numpy(vel.reshape(-1, 3)).pin_memory()
        f = fresh()
        hout = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in f.items()} if rank == 0 else {}

        def e2e_step():
            xp = hpos.to(dev, non_blocking=True)
            xv = hvel.to(dev, non_blocking=True)
            for t in f.values():
                t.zero_()
            voxels_sharded(f, (n_grid,) * 3, BOX, xp, xv, block_dims=(n_part,) * 3, periodic_box=BOX,
                           precision=head)
            for k, t in hout.items():
                t.copy_(f[k], non_blocking=True)
            torch.cuda.synchronize()

        e2e_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        barrier()
        e2e_s = (time.perf_counter() - t0) / args.e2e_steps
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
        field_bytes = sum(v.nbytes for v in f.values())
        e2e = {"value": tets_per_step / e2e_s, "unit": "tets/s", "h2d_bytes_per_step": pos.nbytes + vel.nbytes,
               "d2h_bytes_per_step": field_bytes, "api": f"pypsi_b200.parallel.voxels_sharded(..., precision="
               f"'{head}') over {world} GPUs, mesh from pinned host memory, rank 0 reads the fields back",
               "ms_per_step": e2e_s * 1e3}
        del f, hout
    elif not args.no_e2e:
        mesh = PSI.Mesh(loader="block", pos=pos, vel=vel, periodic_box=BOX)
        grid = PSI.Grid(n=(n_grid,) * 3, bounds=BOX, fields=FIELDS)
        PSI.voxels(grid=grid, mesh=mesh, precision=head)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            PSI.voxels(grid=grid, mesh=mesh, precision=head)
        e2e_s = (time.perf_counter() - t0) / args.e2e_steps
        if dist:
            t = torch.tensor([e2e_s], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        field_bytes = sum(a.nbytes for a in grid.fields.values())
        e2e = {"value": world * tets_per_step / e2e_s, "unit": "tets/s",
               "h2d_bytes_per_step": pos.nbytes + vel.nbytes + mesh.mass.nbytes + field_bytes,
               "d2h_bytes_per_step": field_bytes,
               "api": f"PSI.voxels(grid, mesh, precision='{head}') on host numpy arrays",
               "ms_per_step": e2e_s * 1e3}
        del grid
    # forward + backward of a density loss against forward alone (FP64 forward,
    # adjoint kernel backward) at this workload's sizes and at 64^3 -> 128^3
    adjoint = None
    if not args.no_adjoint and not sharded:
        adjoint = {"forward": "FP64 m field (deposit_density)", "loss": "sum((m/dV - rho_target)^2)",
                   "backward": "psib_voxels_adjoint through torch.autograd (dL/dpos)"}
        sizes = [(n_part, n_grid, RMS, dpos)]
        if (n_part, n_grid) != (64, 128):
            p4, _ = zeldovich(64, 1.0, 4321 + rank)
            sizes.append((64, 128, 1.0, torch.from_numpy(p4.reshape(-1, 3)).to(dev)))
        for npc, ngc, rms, xp in sizes:
            r = time_fwd_bwd(xp, npc, ngc, args.steps, args.warmup, barrier)
            adjoint[f"{npc}^3->{ngc}^3 rms {rms:g}"] = r
        del sizes
        torch.cuda.empty_cache()
    capi.lib.psib_release_device_memory()

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return

    # roofline of the clip walk (its init, level and leaf kernels plus the small
    # deep-tree kernel), following the per-fragment FP64 work of the
    # algorithm: F_2 = 20 V + 132 (2V - 4) + 520 flop per fragment (V = mean
    # vertices per fragment; clip, reduction, projection and accumulation),
    # over the walk's CUDA-event time, against this GPU's FP64 FMA issue rate
    # measured live.  The mixed kernel does the clip term (20 V) in FP32: it is
    # reported against the FP32 rate beside it.  The HBM entry counts the bytes
    # the walk moves by its own algorithm (walk_bytes).
    s = st_mixed[-1]
    frags = s["fragments"] / s["passes"]
    vbar = s["frag_verts"] / max(1, s["fragments"])
    flops = frags * (20 * vbar + 132 * (2 * vbar - 4) + 520)
    flops32 = frags * 20 * vbar
    clip_ms = statistics.mean(x["ms_clip"] for x in st_mixed)
    launches = s["clip_launches"]
    tflops = flops / (clip_ms * 1e-3) / 1e12
    tflops32 = flops32 / (clip_ms * 1e-3) / 1e12
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        peaks = {}
    hbm_peak = peaks.get("hbm_gbs") or 6650.0
    walk_gbs = s["walk_bytes"] / (clip_ms * 1e-3) / 1e9
    value = (1 if sharded else world) * tets_per_step / (ms_mixed * 1e-3)
    traffic = clip_traffic_bytes(frags)
    line = {
        "metric": METRIC, "value": value, "unit": "tets/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True,
        "scaling": "strong" if sharded else "weak",
        "vs_baseline": None, "dtype": "f64" if head == "fp64" else "f32+f64", "data": DATA,
        "config": arm_config(n_part, n_grid, world),
        "precision": "fp64 (reference operation order)" if head == "fp64" else
                     "mixed (FP32 clip, FP64 moments/accumulation)",
        "voxel_clips_per_s": (1 if sharded else world) * frags / (ms_mixed * 1e-3),
        "mixed_vs_fp64_err": {f: e["norm"] for f, e in errs.items() if f != "dead_m"} if errs else None,
        "mixed_vs_fp64_err_m_rel": errs["m"]["rel"] if errs else None,
        "mixed_vs_fp64central_err": {f: e["norm"] for f, e in errs_x.items() if f != "dead_m"} if errs_x else None,
        "fp64_vs_fp64central_err": {f: e["norm"] for f, e in errs_rx.items() if f != "dead_m"} if errs_rx else None,
        "mixed_within_1e5_plus_reference_rounding": within,
        "mass_err": merr,
        "adjoint": adjoint,
        "stage_ms": {"tessellate_and_order": statistics.mean(x["ms_tess"] for x in st_mixed),
                     "clip": statistics.mean(x["ms_clip"] for x in st_mixed),
                     "sort_and_apply": statistics.mean(x["ms_final"] for x in st_mixed)},
        "work": {"tets": tets_per_step, "tet_images": s["tet_images"], "fragments_per_pass": frags,
                 "verts_per_fragment": vbar, "passes": s["passes"], "splits_per_pass": s["splits"] / s["passes"],
                 "mass_corrected_images": s.get("corrected_items")},
        "roofline": {"bound": "fp64", "achieved": tflops, "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": tflops / fp64_peak,
                     "traffic": traffic["bytes_per_step"] if traffic else None,
                     "kernel": "clip walk (its init, level and leaf kernels, and the deep-tree kernel), all launches "
                               "of one step",
                     "achieved_def": "F_2 = 20 V + 132 (2V - 4) + 520 algorithmic flop per fragment x fragments per "
                                     "step / clip CUDA-event time per step",
                     "units": {"fragments_per_step": frags, "verts_per_fragment": vbar,
                               "flop_per_fragment": 20 * vbar + 132 * (2 * vbar - 4) + 520},
                     "peak_source": f"measured live on this GPU: FMA-chain probe (psib_measure_fma_peak), "
                                    f"{fp64_peak:.1f} TFLOP/s FP64; the measured-peaks file has no FP64 figure",
                     "traffic_def": traffic["def"] if traffic else "no capture recorded",
                     "traffic_over_algorithmic": (traffic["bytes_per_step"] / (frags * ALG_BYTES_PER_FRAGMENT)
                                                  if traffic else None),
                     "fp32": {"achieved": tflops32, "peak": fp32_peak, "unit": "TFLOP/s", "frac": tflops32 / fp32_peak,
                              "def": "clip term 20 V flop per fragment (FP32 in the mixed kernel) / clip time; peak "
                                     "measured live by the same probe in FP32"},
                     "hbm": {"achieved": walk_gbs, "peak": hbm_peak, "unit": "GB/s", "frac": walk_gbs / hbm_peak,
                             "def": "walk_bytes (polyhedra read and written between levels, tet vertices, records, "
                                    "counted by the kernels) / clip time; peak MEASURED_PEAKS.json hbm_gbs"
                                    + (" (of measured)" if peaks.get("hbm_gbs") else " (fallback)")},
                     "clip_ms_per_step": clip_ms, "clip_launches_per_step": launches},
        "e2e": e2e,
        "gpu_launches": int(sum(x["kernel_launches"] for x in st_mixed)),
        "clocks": clocks,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"], ref_slab = cpu_baseline_single()

        def deposit(n, bounds, prec):
            f = {k: torch.zeros(n + sh[3:], dtype=torch.float64, device=dev) for k, sh in shapes.items()}
            step(f, prec, n, bounds)
            return {k: v.cpu().numpy() for k, v in f.items()}

        line["parity_vs_reference"] = parity_on_slab(ref_slab, deposit)
        capi.lib.psib_release_device_memory()
    # the other workloads the target names, compact, on one GPU (--no-extra skips them)
    if world == 1 and not args.no_extra and (n_part, n_grid) == (N_PART, N_GRID):
        c3 = c3_result(args, 2, 1)
        line["c3_batch"] = {k: c3[k] for k in ("value", "unit", "ms_per_step", "batch_over_separate",
                                               "separate_calls", "graph_replay", "autotuned", "work")}
        c5 = c5_result(args, 2, 1)
        line["c5_refined"] = {k: c5[k] for k in ("value", "unit", "ms_per_step", "mass_err_mixed", "work")}
    # the comparison the metric names, last so that the tail of the line shows it
    line["fp64"] = {"value": (1 if sharded else world) * tets_per_step / (ms_fp64 * 1e-3), "unit": "tets/s",
                    "ms_per_step": ms_fp64,
                    "walk": "breadth-first" if st_fp64 and st_fp64[-1]["walk_bytes"] > 0 else "depth-first"}
    line["mixed_over_fp64"] = ms_fp64 / ms_mixed
    line["fwd_bwd_over_fwd"] = adjoint[f"{n_part}^3->{n_grid}^3 rms {RMS:g}"]["ratio"] if adjoint else None
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "loaders":
        run_loaders(args)
    elif args.impl == "reference" and args.workload == "ann":
        run_reference_ann(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "ann":
        run_ann(args)
    elif args.workload == "vdf":
        run_vdf(args)
    elif args.workload == "quad":
        run_quad(args)
    elif args.workload == "c5":
        run_c5(args)
    elif args.workload == "c3":
        run_c3(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
