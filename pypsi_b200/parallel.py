"""One mesh deposited by several GPUs: element slabs and the field exchange.

Tets are independent, so the deposit shards over the Lagrangian element index
space: rank r of W voxelizes the contiguous slab of elements
``element_slab(nelem, W, r)`` into a full-size grid of its own, and one
exchange step combines the ranks' grids on every rank.  The combination is the
merge of the reference's online update (src/geometry.c:164-186) applied to W
partial results at once:

    M  = sum_r M_r
    X  = sum_r M_r X_r / M                       (V alike)
    XX = sum_r M_r (XX_r + (X_r - X)(X_r - X)^T) / M   (XV with V, VV alike)

taken in two all-reduces (first M, M X, M V; then the second moments about
the global means, so nothing cancels).  The sums run in a different order
from a single deposit, so FP64 results agree with it to rounding, not bit for
bit.  The collectives are torch.distributed all-reduces: NCCL over NVLink for
CUDA tensors, gloo for CPU tensors.
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


def merge_fields(fields: dict, group=None) -> dict:
    """Combine every rank's partial fields (m, and any of x, v, xx, xv, vv, in
    the reference's layout) into the fields of the whole mesh, in place, on
    every rank of `group`."""
    m = fields["m"]
    first = [f for f in ("x", "v") if f in fields]
    # pass 1: M and the mass-weighted first moments
    buf1 = [m.clone()] + [fields[f] * m.unsqueeze(-1) for f in first]
    for b in buf1:
        dist.all_reduce(b, group=group)
    mt = buf1[0]
    safe = torch.where(mt > 0, mt, torch.ones_like(mt))
    means = {f: b / safe.unsqueeze(-1) for f, b in zip(first, buf1[1:])}
    # pass 2: second moments about the global means
    second = [f for f in ("xx", "xv", "vv") if f in fields]
    buf2 = []
    for f in second:
        a, b = SECOND[f]
        da = fields[a] - means[a]
        db = fields[b] - means[b]
        buf2.append((fields[f] + da.unsqueeze(-1) * db.unsqueeze(-2)) * m[..., None, None])
    for b in buf2:
        dist.all_reduce(b, group=group)
    for f, b in zip(second, buf2):
        fields[f].copy_(torch.where(mt[..., None, None] > 0, b / safe[..., None, None], torch.zeros_like(b)))
    for f in first:
        fields[f].copy_(torch.where(mt.unsqueeze(-1) > 0, means[f], torch.zeros_like(means[f])))
    fields["m"].copy_(mt)
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
