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
