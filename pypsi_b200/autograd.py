"""Differentiable deposits: ``torch.autograd.Function`` over the C ABI.

``deposit_density(pos, mass, n=..., bounds=..., ...)`` returns the m field of
``PSI.voxels`` (mass per voxel, float64, shape n) for particle positions held
in a CUDA tensor.  Its backward pass is ``psib_voxels_adjoint``: the clip is
recomputed in FP64 and each fragment's mass fraction is differentiated through
the fragment faces that lie on the faces of its tet.  Gradients flow to the
positions and, when it requires them, to the element masses.  The m field does
not depend on velocities, so none are taken.

``deposit_fields(pos, vel, mass, fields=(...), ...)`` returns every requested
field -- m, x, v, xx, xv, vv, as PSI.voxels leaves them in a zeroed grid -- and
its backward pass, ``psib_voxels_adjoint_fields``, gives the gradients with
respect to positions, velocities and element masses through all of them.

PyPSI itself is not differentiable; the forward pass is its density branch
(src/cpsi.c:41-112, src/geometry.c:60-188), computed by ``psib_voxels``.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from . import capi


@dataclass(frozen=True)
class DepositSpec:
    """The grid and the mesh topology of a deposit (everything but the tensors)."""

    n: tuple
    bounds: tuple
    block_dims: tuple | None = None
    periodic_box: tuple | None = None
    precision: str = "fp64"
    refine_tolerance: float = 1.0
    refine_max_lvl: int = 0


class _DensityDeposit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, mass, connectivity, spec: DepositSpec):
        m = torch.zeros(spec.n, dtype=torch.float64, device=pos.device)
        capi.voxels_device({"m": m}, spec.n, spec.bounds, pos, None, mass, connectivity=connectivity,
                           block_dims=spec.block_dims, periodic_box=spec.periodic_box, precision=spec.precision,
                           refine_tolerance=spec.refine_tolerance, refine_max_lvl=spec.refine_max_lvl)
        ctx.save_for_backward(pos, mass, connectivity)
        ctx.spec = spec
        return m

    @staticmethod
    def backward(ctx, grad_m):
        pos, mass, connectivity = ctx.saved_tensors
        spec = ctx.spec
        grad_pos = torch.zeros_like(pos)
        grad_mass = torch.zeros_like(mass) if (mass is not None and ctx.needs_input_grad[1]) else None
        capi.adjoint_device(grad_m.contiguous(), spec.n, spec.bounds, pos, grad_pos, mass=mass,
                            connectivity=connectivity, block_dims=spec.block_dims,
                            periodic_box=spec.periodic_box, grad_mass=grad_mass,
                            refine_tolerance=spec.refine_tolerance, refine_max_lvl=spec.refine_max_lvl)
        return (grad_pos if ctx.needs_input_grad[0] else None), grad_mass, None, None


def deposit_density(pos: torch.Tensor, mass: torch.Tensor | None = None, *, n, bounds, block_dims=None,
                    connectivity: torch.Tensor | None = None, periodic_box=None,
                    precision: str = "fp64", refine_tolerance: float = 1.0,
                    refine_max_lvl: int = 0) -> torch.Tensor:
    """m field of PSI.voxels(grid, mesh) for particles at `pos`, differentiable.

    pos: (npart, 3) float64 CUDA tensor (C-contiguous).  mass: (nelem,) float64
    or None (1 per element).  The mesh is a block lattice (`block_dims`, as
    Mesh(loader='block')) or explicit `connectivity` ((nelem, 4|8) int32), in a
    periodic box when `periodic_box` is given.  `precision` selects the forward
    kernel ('fp64' or 'mixed'); the backward pass is always FP64.  Elements are
    refined as PSI.voxels refines them (midpoint criterion); the gradient flows
    through the interpolation of the refined vertices."""
    if not pos.is_cuda:
        raise ValueError("deposit_density runs on the GPU: pos must be a CUDA tensor")
    if pos.dtype != torch.float64 or not pos.is_contiguous():
        raise ValueError("pos must be a C-contiguous float64 tensor")
    if mass is not None and (mass.dtype != torch.float64 or not mass.is_contiguous()):
        raise ValueError("mass must be a C-contiguous float64 tensor")
    if connectivity is None and block_dims is None:
        raise ValueError("give block_dims or connectivity")
    spec = DepositSpec(tuple(int(v) for v in n), tuple(tuple(float(x) for x in b) for b in bounds),
                       tuple(int(v) for v in block_dims) if block_dims is not None else None,
                       tuple(tuple(float(x) for x in b) for b in periodic_box) if periodic_box is not None else None,
                       precision, float(refine_tolerance), int(refine_max_lvl))
    return _DensityDeposit.apply(pos, mass, connectivity, spec)


FIELD_SHAPES = {"m": (), "x": (3,), "v": (3,), "xx": (3, 3), "xv": (3, 3), "vv": (3, 3)}
FIELD_ORDER = ("m", "x", "v", "xx", "xv", "vv")


class _FieldsDeposit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, vel, mass, connectivity, spec: DepositSpec, names: tuple):
        out = {f: torch.zeros(spec.n + FIELD_SHAPES[f], dtype=torch.float64, device=pos.device) for f in names}
        capi.voxels_device(out, spec.n, spec.bounds, pos, vel, mass, connectivity=connectivity,
                           block_dims=spec.block_dims, periodic_box=spec.periodic_box, precision=spec.precision,
                           deterministic=True, refine_tolerance=spec.refine_tolerance,
                           refine_max_lvl=spec.refine_max_lvl)
        res = tuple(out[f] for f in names)
        ctx.save_for_backward(pos, vel, mass, connectivity, *res)
        ctx.spec = spec
        ctx.names = names
        return res

    @staticmethod
    def backward(ctx, *grads):
        pos, vel, mass, connectivity, *res = ctx.saved_tensors
        spec, names = ctx.spec, ctx.names
        fwd = dict(zip(names, res))
        g = {f: t.contiguous() for f, t in zip(names, grads) if t is not None}
        grad_pos = torch.zeros_like(pos)
        grad_vel = torch.zeros_like(vel) if (vel is not None and ctx.needs_input_grad[1]) else None
        grad_mass = torch.zeros_like(mass) if (mass is not None and ctx.needs_input_grad[2]) else None
        if g:
            capi.adjoint_fields_device(g, fwd, spec.n, spec.bounds, pos, grad_pos, vel=vel, mass=mass,
                                       connectivity=connectivity, block_dims=spec.block_dims,
                                       periodic_box=spec.periodic_box, grad_vel=grad_vel, grad_mass=grad_mass,
                                       refine_tolerance=spec.refine_tolerance, refine_max_lvl=spec.refine_max_lvl)
        return (grad_pos if ctx.needs_input_grad[0] else None), grad_vel, grad_mass, None, None, None


def deposit_fields(pos: torch.Tensor, vel: torch.Tensor | None = None, mass: torch.Tensor | None = None, *,
                   fields=("m",), n, bounds, block_dims=None, connectivity: torch.Tensor | None = None,
                   periodic_box=None, refine_tolerance: float = 1.0, refine_max_lvl: int = 0) -> dict:
    """The requested fields of PSI.voxels(grid, mesh) in a zeroed grid --
    m (mass), x and v (mass-weighted means), xx, xv, vv ((co)variances, xv with
    the reference's pairing of its cross terms) -- differentiable with respect
    to pos, vel ((npart, 3) float64 CUDA tensors) and mass ((nelem,)).

    The forward pass is the FP64 deposit in the reference's order; the
    backward pass recomputes the clip in FP64 (psib_voxels_adjoint_fields).
    A second moment needs its first moments among `fields`.  Elements are refined
    as PSI.voxels refines them (midpoint criterion, 8- and 27-node elements); the
    gradient flows through the interpolation of the refined vertices.  Returns
    {name: tensor} for the requested names (m always included)."""
    for t, name in ((pos, "pos"), (vel, "vel"), (mass, "mass")):
        if t is not None and (not t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous()):
            raise ValueError(f"{name} must be a C-contiguous float64 CUDA tensor")
    if connectivity is None and block_dims is None:
        raise ValueError("give block_dims or connectivity")
    names = tuple(f for f in FIELD_ORDER if f == "m" or f in fields)
    if vel is None and any(f in names for f in ("v", "xv", "vv")):
        vel = torch.zeros_like(pos)
    spec = DepositSpec(tuple(int(v) for v in n), tuple(tuple(float(x) for x in b) for b in bounds),
                       tuple(int(v) for v in block_dims) if block_dims is not None else None,
                       tuple(tuple(float(x) for x in b) for b in periodic_box) if periodic_box is not None else None,
                       "fp64", float(refine_tolerance), int(refine_max_lvl))
    res = _FieldsDeposit.apply(pos, vel, mass, connectivity, spec, names)
    return dict(zip(names, res))
