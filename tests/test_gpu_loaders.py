"""A deposit from a loaded snapshot, the reference tutorial's sequence
(PSI.Mesh(loader='gadget2'), a Grid over mesh.wrapbox with fields v and vv,
PSI.voxels with refinement), on a synthetic Gadget-2 / gevolution snapshot:
FP64 equals the reference (compiled, or the oracle's restatement pinned to
it) bit for bit, mixed precision is within
1e-5 of it, and the total mass is conserved."""
import numpy as np
import pytest

from pypsi_b200.metrics import field_errors, mass_error
from snapshots import make_snapshot

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("flavour", ["gadget2", "gevolution"])
def test_snapshot_deposit(gpu, oracle, tmp_path, flavour):
    path = str(tmp_path / "snap")
    make_snapshot(path, 8, flavour=flavour, seed=3)
    mesh = gpu.Mesh(loader=flavour, filename=path)
    kw = dict(refine_max_lvl=1, refine_tolerance=0.1)
    # the compiled reference where it travelled with the tree, else the restatement pinned to it
    kind = "reference" if oracle.available("reference") else "restatement"
    ref = oracle.voxelize(kind, (24, 24, 24), mesh.wrapbox, mesh.pos, mesh.connectivity, vel=mesh.vel,
                          mass=mesh.mass, periodic_box=mesh.wrapbox, fields=("v", "vv"), reftol=0.1, maxlvl=1)
    grid = gpu.Grid(n=(24, 24, 24), bounds=mesh.wrapbox, fields=["v", "vv"])
    gpu.voxels(grid=grid, mesh=mesh, **kw)
    for f in ref:
        assert np.array_equal(grid.fields[f], ref[f]), (flavour, f)
    assert mass_error(grid.fields["m"], float(np.sum(mesh.mass))) <= 1e-13
    mixed = gpu.Grid(n=(24, 24, 24), bounds=mesh.wrapbox, fields=["v", "vv"])
    gpu.voxels(grid=mixed, mesh=mesh, precision="mixed", **kw)
    errs = field_errors(dict(mixed.fields), ref)
    assert errs["m"]["rel"] <= 1e-5, errs["m"]
    assert mass_error(mixed.fields["m"], float(np.sum(mesh.mass))) <= 1e-13
