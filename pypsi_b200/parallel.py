"""One mesh deposited by several GPUs: element slabs and the field exchange.

Tets are independent, so the deposit shards over the Lagrangian element index
space: rank r of W voxelizes the contiguous slab of elements
``element_slab(nelem, W, r)`` into a full-size grid of its own, and one
exchange step combines the ranks' grids.  The combination is the merge of the
reference's online update (src/geometry.c:164-186) applied to W partial
results at once:

    M  = sum_r M_r
    X  = sum_r M_r X_r / M                       (V alike)
    XX = sum_r M_r (XX_r + (X_r - X)(X_r - X)^T) / M   (XV with V, VV alike)

The exchange sends raw sums, so that it is one reduction: each rank turns its
fields into per-voxel sums about reference points c (position) and u
(velocity) --

    S0 = M_r,  Sx = M_r (X_r - c),  Sv = M_r (V_r - u),
    Sxx = M_r (XX_r + (X_r - c)(X_r - c)^T),  Sxv, Svv alike --

one reduce-scatter adds them over the ranks, each rank getting a slab of voxel
planes along the first axis, and each rank turns its slab back into M, X, V
and (co)variances; an all-gather of the finished slabs gives every rank the
whole grid.  c and u must be the same on every rank and close to the voxel's
final means, or Sxx / M - (Sx / M)(Sx / M)^T cancels in voxels made of tiny
fragments: they are the means to single precision, from one all-reduce of
M, M X and M V in FP32 (7 floats per voxel, against 34 doubles in the
reduce-scatter).  The sums run in a different order from a single deposit, so
FP64 results agree with it to rounding, not bit for bit.  The collectives are
torch.distributed: NCCL over NVLink for CUDA tensors (reduce_scatter_tensor,
all_gather_into_tensor), gloo for CPU tensors (which has no reduce-scatter: an
all-reduce, then the rank's slab).
"""
from __future__ import annotations

import torch
import torch.distributed as dist

SECOND = {"xx": ("x", "x"), "xv": ("x", "v"), "vv": ("v", "v")}


def element_slab(nelem: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous element range [e0, e1) of `rank`: sizes differ by at most one."""
    base, extra = divmod(int(nelem), int(world))
    e0 = rank * base + min(rank, extra)
    return e0, e0 + base + (1 if rank < extra else 0)


def block_slab_connectivity(block_dims, periodic: bool, e0: int, e1: int, device=None) -> torch.Tensor:
    """Connectivity rows [e0, e1) of a block mesh, as Mesh(loader='block') builds
    them (src/PSI.c:636-656): element (i,j,k) -> particles of corners 4ii+2jj+kk."""
    nx, ny, nz = (int(v) for v in block_dims)
    ex, ey, ez = (nx, ny, nz) if periodic else (nx - 1, ny - 1, nz - 1)
    e = torch.arange(e0, e1, dtype=torch.int64, device=device)
    i, j, k = e // (ey * ez), (e // ez) % ey, e % ez
    cols = []
    for ii in range(2):
        for jj in range(2):
            for kk in range(2):
                cols.append(ny * nz * ((i + ii) % nx) + nz * ((j + jj) % ny) + (k + kk) % nz)
    return torch.stack(cols, dim=1).to(torch.int32).contiguous()


def _is_nccl(group) -> bool:
    return dist.get_backend(group) == "nccl"


def _reduce_scatter_rows(buf: torch.Tensor, world: int, rank: int, group) -> torch.Tensor:
    """Sum of buf over the ranks, rank's slab of rows (buf.shape[0] divisible by world)."""
    rows = buf.shape[0] // world
    if _is_nccl(group):
        out = torch.empty((rows,) + tuple(buf.shape[1:]), dtype=buf.dtype, device=buf.device)
        dist.reduce_scatter_tensor(out, buf.contiguous(), group=group)
        return out
    dist.all_reduce(buf, group=group)
    return buf[rank * rows:(rank + 1) * rows].clone()


def _all_gather_rows(part: torch.Tensor, world: int, group) -> torch.Tensor:
    if _is_nccl(group):
        out = torch.empty((world * part.shape[0],) + tuple(part.shape[1:]), dtype=part.dtype, device=part.device)
        dist.all_gather_into_tensor(out, part.contiguous(), group=group)
        return out
    parts = [torch.empty_like(part) for _ in range(world)]
    dist.all_gather(parts, part.contiguous(), group=group)
    return torch.cat(parts)


def merge_fields(fields: dict, group=None) -> dict:
    """Combine every rank's partial fields (m, and any of x, v, xx, xv, vv, in
    the reference's layout) into the fields of the whole mesh, in place, on
    every rank of `group`."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    m = fields["m"]
    n = tuple(m.shape)
    dev, dt = m.device, m.dtype
    hx, hv = "x" in fields, "v" in fields
    second = [f for f in ("xx", "xv", "vv") if f in fields]
    # reference points, equal on every rank: the merged means in single precision
    c = u = None
    if hx or hv:
        parts = [m.unsqueeze(-1)] + [m.unsqueeze(-1) * fields[f] for f in ("x", "v") if f in fields]
        approx = torch.cat(parts, dim=-1).float()
        dist.all_reduce(approx, group=group)
        mt = approx[..., :1]
        means = (approx[..., 1:] / torch.where(mt > 0, mt, torch.ones_like(mt))).to(dt)
        if hx:
            c = means[..., :3]
        if hv:
            u = means[..., 3:6] if hx else means[..., :3]
    # raw sums, (voxel, component), padded to a multiple of `world` voxel planes
    comps = [m.unsqueeze(-1)]
    dx = fields["x"] - c if hx else None
    dv = fields["v"] - u if hv else None
    if hx:
        comps.append(m.unsqueeze(-1) * dx)
    if hv:
        comps.append(m.unsqueeze(-1) * dv)
    for f in second:
        a, b = SECOND[f]
        da = dx if a == "x" else dv
        db = dx if b == "x" else dv
        comps.append((m[..., None, None] * (fields[f] + da.unsqueeze(-1) * db.unsqueeze(-2))).reshape(n + (9,)))
    raw = torch.cat(comps, dim=-1)
    rows = (n[0] + world - 1) // world
    buf = torch.zeros((rows * world,) + n[1:] + (raw.shape[-1],), dtype=dt, device=dev)
    buf[: n[0]] = raw
    del raw, comps
    part = _reduce_scatter_rows(buf, world, rank, group)
    del buf
    # this rank's slab of voxel planes back to fields
    i0 = rank * rows
    i1 = min(i0 + rows, n[0])
    S = part[: max(0, i1 - i0)]
    s0 = S[..., 0]
    live = s0 > 0
    safe = torch.where(live, s0, torch.ones_like(s0))
    out = {"m": s0}
    k = 1
    mx = mv = None
    if hx:
        mx = S[..., k:k + 3] / safe.unsqueeze(-1)
        out["x"] = torch.where(live.unsqueeze(-1), c[i0:i1] + mx, torch.zeros_like(mx))
        k += 3
    if hv:
        mv = S[..., k:k + 3] / safe.unsqueeze(-1)
        out["v"] = torch.where(live.unsqueeze(-1), u[i0:i1] + mv, torch.zeros_like(mv))
        k += 3
    for f in second:
        a, b = SECOND[f]
        ma = mx if a == "x" else mv
        mb = mx if b == "x" else mv
        cov = S[..., k:k + 9].reshape(S.shape[:3] + (3, 3)) / safe[..., None, None] - ma.unsqueeze(-1) * mb.unsqueeze(-2)
        out[f] = torch.where(live[..., None, None], cov, torch.zeros_like(cov))
        k += 9
    # every rank gets the whole grid
    for f, slab in out.items():
        pad = torch.zeros((rows,) + tuple(slab.shape[1:]), dtype=dt, device=dev)
        pad[: slab.shape[0]] = slab
        fields[f].copy_(_all_gather_rows(pad, world, group)[: n[0]])
    return fields


def voxels_sharded(fields: dict, n, bounds, pos, vel=None, mass=None, block_dims=None, connectivity=None,
                   periodic_box=None, precision="fp64", group=None, refine_tolerance=1.0, refine_max_lvl=0) -> dict:
    """PSI.voxels of one mesh on all ranks of `group`, one GPU each.

    Every rank passes the whole mesh (device tensors) and zeroed fields; it
    deposits its element slab through the C ABI, then the ranks exchange.
    Returns the fields, equal on every rank."""
    from . import capi

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if connectivity is None:
        nelem = 1
        for b in block_dims:
            nelem *= b if periodic_box is not None else b - 1
    else:
        nelem = connectivity.shape[0]
    e0, e1 = element_slab(nelem, world, rank)
    if connectivity is None:
        conn = block_slab_connectivity(block_dims, periodic_box is not None, e0, e1, device=pos.device)
    else:
        conn = connectivity[e0:e1].contiguous()
    slab_mass = None if mass is None else mass.reshape(-1)[e0:e1].contiguous()
    if e1 > e0:
        capi.voxels_device(fields, n, bounds, pos, vel, slab_mass, connectivity=conn, periodic_box=periodic_box,
                           precision=precision, refine_tolerance=refine_tolerance, refine_max_lvl=refine_max_lvl)
    return merge_fields(fields, group)


# ---- annihilation: split by grid window ----
# Annihilation pairs elements across any element slab, so it splits by grid
# window instead: rank r deposits voxel planes [i0, i1) along axis 0 -- a
# sub-window of the grid -- with the whole mesh (an element whose box misses
# the sub-window is culled, and every pair that reaches the sub-window's voxels
# has both elements there), and the ranks gather the slabs.  A voxel's value is
# the same sum in the same order as on one GPU; only the window planes the
# fragments are cut by differ at the slab edges, to rounding.  Open meshes
# only: the reference refines a pair's partner from its stored vertices
# (src/cpsi.c:123-131), so in a periodic mesh a partner that wraps the box edge
# reaches voxels far from its unwrapped box, and a slab's cull would drop it.

def window_slab(n, bounds, world: int, rank: int):
    """Voxel planes [i0, i1) along axis 0 of `rank`, the slab's grid size and its
    bounds (the full grid's voxel size d on every axis)."""
    i0, i1 = element_slab(int(n[0]), world, rank)
    d0 = (float(bounds[1][0]) - float(bounds[0][0])) / int(n[0])
    lo = (float(bounds[0][0]) + i0 * d0,) + tuple(float(v) for v in bounds[0][1:])
    hi = (float(bounds[0][0]) + i1 * d0,) + tuple(float(v) for v in bounds[1][1:])
    return i0, i1, (i1 - i0,) + tuple(int(v) for v in n[1:]), (lo, hi)


def _gather_rows(local: torch.Tensor, group=None) -> list:
    """All ranks' tensors (of equal trailing shape, any length along axis 0), on every rank."""
    world = dist.get_world_size(group)
    size = torch.tensor([local.shape[0]], dtype=torch.int64, device=local.device)
    sizes = [torch.zeros_like(size) for _ in range(world)]
    dist.all_gather(sizes, size, group=group)
    sizes = [int(s.item()) for s in sizes]
    top = max(sizes) if sizes else 0
    pad = torch.zeros((top,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.zeros_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return [p[:s] for p, s in zip(parts, sizes)]


def gather_window_slabs(m: torch.Tensor, local: torch.Tensor, group=None) -> torch.Tensor:
    """Add every rank's slab of voxel planes (window_slab) into the full field m,
    on every rank of `group`; returns m."""
    world = dist.get_world_size(group)
    for r, part in enumerate(_gather_rows(local, group)):
        i0, i1 = element_slab(m.shape[0], world, r)
        m[i0:i1] += part
    return m


def annihilation_sharded(m: torch.Tensor, n, bounds, pos, connectivity=None, block_dims=None, mass=None,
                         periodic_box=None, refine_tolerance=1.0, refine_max_lvl=0, group=None) -> torch.Tensor:
    """PSI.voxels(mode='annihilation') of one open mesh on all ranks of `group`,
    one GPU each: every rank passes the whole mesh and its full m field (device
    tensors); it deposits its window slab, then the ranks gather.  m gains the
    whole deposit on every rank."""
    from . import capi

    if periodic_box is not None:
        raise NotImplementedError("annihilation splits by grid window for open meshes only: a periodic mesh's "
                                  "wrapped partner elements reach past any window slab")
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    i0, i1, sub_n, sub_bounds = window_slab(n, bounds, world, rank)
    local = torch.zeros(sub_n, dtype=torch.float64, device=m.device)
    if i1 > i0:
        capi.voxels_device({"m": local}, sub_n, sub_bounds, pos, None, mass, connectivity=connectivity,
                           block_dims=block_dims, periodic_box=periodic_box, refine_tolerance=refine_tolerance,
                           refine_max_lvl=refine_max_lvl, mode="annihilation")
    return gather_window_slabs(m, local, group)


# ---- phase-space samples: split by points ----

def gather_samples(offsets: torch.Tensor, rho: torch.Tensor, vel: torch.Tensor, group=None):
    """Join every rank's samples of its slab of points (element_slab over the
    points) into the samples of all points, in point order, on every rank:
    (offsets (npoints + 1,), rho, vel) as psib_sample_vdf returns them."""
    counts = offsets[1:] - offsets[:-1]
    all_counts = torch.cat(_gather_rows(counts, group))
    all_rho = torch.cat(_gather_rows(rho, group))
    all_vel = torch.cat(_gather_rows(vel, group))
    off = torch.zeros(all_counts.shape[0] + 1, dtype=torch.int64, device=offsets.device)
    off[1:] = torch.cumsum(all_counts, 0)
    return off, all_rho, all_vel


def sample_vdf_sharded(points, pos, group=None, **kw):
    """capi.sample_vdf of all points on all ranks of `group`: rank r samples its
    slab of the points on its GPU, then the ranks gather (no reduction)."""
    from . import capi

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    p0, p1 = element_slab(points.shape[0], world, rank)
    off, rho, vel = capi.sample_vdf(points[p0:p1], pos, **kw)
    return gather_samples(off, rho, vel, group)
