"""GPU parity against the CPU oracle, through the drop-in PSI module (which
calls the C ABI of libpsi_b200.so).

Bounds (from the target spec): per-voxel relative error <= 1e-12 for the FP64
kernel and <= 1e-5 for the mixed-precision kernel, total deposited mass equal
to the particle mass to 1e-13 relative.  The per-voxel bound is applied to m
strictly and to every field in the voxel-scale normalisation of
pypsi_b200.metrics ("norm"); the deterministic mode must equal the reference
bit for bit.

The reference's own FP64 result carries rounding error of up to ~1e-4 in the
second moments of voxels made of tiny fragments (their raw q-moments about the
tet's vertex 0 cancel).  The mixed and FP64-central results are therefore
checked against the exact result of the same algorithm (the oracle in quad
precision), and against the reference within the bound plus the reference's
own error in each voxel.
"""
import os

import numpy as np
import pytest

from cases import NAMES, load_golden, make, run_oracle, run_psi, total_mass
from pypsi_b200.metrics import error_maps, field_errors, mass_error

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-5
MASS_TOL = 1e-13
FULL_BOX = {"c1_small", "c2_small", "c2_order1", "rms3_vvonly", "lattice", "refine", "big_tet", "tets"}

_ref_cache = {}
_exact_cache = {}


def reference(oracle, name):
    if name not in _ref_cache:
        _ref_cache[name] = run_oracle(oracle, make(name), counters=True)
    return _ref_cache[name]


def _exact_one(name):
    import oracle as O

    return name, run_oracle(O, make(name), kind="exact")


def exact(oracle, name):
    """The oracle in quad precision, for all cases at once on a spawn pool (slow: ~60x FP64)."""
    if not _exact_cache:
        import multiprocessing as mp

        with mp.get_context("spawn").Pool(min(len(NAMES), os.cpu_count() or 1)) as pool:
            _exact_cache.update(dict(pool.map(_exact_one, NAMES)))
    return _exact_cache[name]


def check_vs_exact_and_reference(out, ref, ex, tol, name):
    """Within tol of the exact result, and within tol plus the reference's own
    error of the reference, voxel by voxel."""
    check(field_errors(out, ex), tol, name)
    e_or = error_maps(out, ref, scale_from=ex)
    e_rx = error_maps(ref, ex)
    for f in e_or:
        bad = e_or[f] > tol + e_rx[f]
        assert not bad.any(), (name, f, float(e_or[f][bad].max()), float(e_rx[f][bad].max()))


def check(errs, tol, name):
    assert errs["m"]["rel"] <= tol, (name, "m", errs["m"])
    for f, e in errs.items():
        if f == "dead_m":
            assert e == 0.0, (name, "mass outside the reference's footprint", e)
        else:
            assert e["norm"] <= tol, (name, f, e)


@pytest.mark.parametrize("name", NAMES)
def test_fp64_matches_oracle(gpu, oracle, name):
    """The FP64 path repeats the reference's arithmetic and update order:
    every field equals the reference's bit for bit (so also within 1e-12)."""
    ref, cnt = reference(oracle, name)
    c = make(name)
    out, _, _ = run_psi(gpu, c, precision="fp64")
    check(field_errors(out, ref), FP64_TOL, name)
    for f in ref:
        assert np.array_equal(out[f], ref[f]), (name, f, np.abs(out[f] - ref[f]).max())
    st = gpu.last_stats()
    assert st["fragments"] == cnt["fragments"]
    assert st["splits"] == cnt["splits"]
    if name in FULL_BOX:
        assert mass_error(out["m"], total_mass(c)) <= MASS_TOL


@pytest.mark.parametrize("name", NAMES)
def test_deterministic_is_bitwise_reference(gpu, oracle, name):
    ref, _ = reference(oracle, name)
    out, _, _ = run_psi(gpu, make(name), precision="fp64", deterministic=True)
    for f in ref:
        assert np.array_equal(out[f], ref[f]), (name, f, np.abs(out[f] - ref[f]).max())


@pytest.mark.parametrize("det", [False, True], ids=["atomic", "sorted"])
@pytest.mark.parametrize("name", NAMES)
def test_mixed_within_1e5(gpu, oracle, name, det):
    """Mixed precision in both accumulation modes: per-voxel FP64 atomic sums
    (the default) and sorted records applied in order (deterministic=True)."""
    ref, _ = reference(oracle, name)
    c = make(name)
    out, _, _ = run_psi(gpu, c, precision="mixed", deterministic=det)
    assert gpu.last_stats()["accumulation"] == (0 if det else 1)
    check_vs_exact_and_reference(out, ref, exact(oracle, name), MIXED_TOL, name)
    if name in FULL_BOX:
        assert mass_error(out["m"], total_mass(c)) <= MASS_TOL


@pytest.mark.parametrize("det", [False, True], ids=["atomic", "sorted"])
@pytest.mark.parametrize("name", NAMES)
def test_fp64_central_near_exact(gpu, oracle, name, det):
    """The FP64 walk with central moments: FP64 accuracy where the reference's
    raw moments lose it, in both accumulation modes."""
    ref, _ = reference(oracle, name)
    c = make(name)
    out, _, _ = run_psi(gpu, c, precision="fp64-central", deterministic=det)
    check_vs_exact_and_reference(out, ref, exact(oracle, name), 1e-9, name)
    if name in FULL_BOX:
        assert mass_error(out["m"], total_mass(c)) <= MASS_TOL


@pytest.mark.parametrize("name", NAMES)
def test_atomic_sums_equal_sorted_records(gpu, name):
    """The atomic mode adds the same fragments as the sorted mode, about
    reference points claimed by each voxel's first fragment instead of the
    run's first fragment: the two agree to rounding, and the FP64 path ignores
    the flag (always the reference's order).

    Rounding here is the level at which two exact orders of the same FP64
    fragments already differ: the reference's own order (fp64) against the
    central merge in sorted order (fp64-central, deterministic).  Second
    moments of voxels whose velocity spread is small against their mean
    velocity lose digits in E[vv] - E[v]E[v] in any order (a few 1e-12 of the
    voxel's scale at these sizes), so the bound is 4x that level, and never
    below 1e-12."""
    c = make(name)
    a, _, _ = run_psi(gpu, c, precision="mixed", deterministic=False)
    b, _, _ = run_psi(gpu, c, precision="mixed", deterministic=True)
    r64, _, _ = run_psi(gpu, c, precision="fp64")
    assert gpu.last_stats()["accumulation"] == 0
    rc, _, _ = run_psi(gpu, c, precision="fp64-central", deterministic=True)
    level = field_errors(rc, r64)
    errs = field_errors(a, b)
    assert errs["m"]["rel"] <= 1e-12 and errs["dead_m"] == 0.0, (name, errs["m"])
    for f, e in errs.items():
        if f != "dead_m":
            assert e["norm"] <= max(1e-12, 4.0 * level[f]["norm"]), (name, f, e, level[f])


@pytest.mark.parametrize("gname", sorted(load_golden()))
@pytest.mark.parametrize("det", [False, True])
def test_golden_fixtures(gpu, gname, det):
    c, exp = load_golden()[gname]
    out, _, _ = run_psi(gpu, c, deterministic=det)
    if det:
        for f in exp:
            assert np.array_equal(out[f], exp[f]), (gname, f)
    else:
        for f in exp:
            assert np.array_equal(out[f], exp[f]), (gname, f)


@pytest.mark.parametrize("det", [False, True])
def test_accumulates_into_existing_grid(gpu, oracle, det):
    """voxels() merges into the fields already on the grid (src/geometry.c:164-186)."""
    a, b = make("c2_small"), make("c2_order1")
    b["fields"] = a["fields"]
    ref = run_oracle(oracle, a)
    ref = oracle.voxelize("restatement", n=b["n"], bounds=b["bounds"], pos=b["pos"].reshape(-1, 3),
                          vel=b["vel"].reshape(-1, 3), conn=oracle.block_connectivity((16, 16, 16), True),
                          periodic_box=b["periodic_box"], fields=b["fields"], out=ref)
    _, grid, _ = run_psi(gpu, a, deterministic=det)
    out, _, _ = run_psi(gpu, b, grid=grid, deterministic=det)
    if det:
        for f in ref:
            assert np.array_equal(out[f], ref[f]), f
    else:
        check(field_errors(out, ref), FP64_TOL, "accumulate")


def test_stretch_refinement_fp64_bitwise_and_mixed(gpu, oracle):
    """The stretch refinement criterion: the same tets as the oracle's
    statement of it, FP64 fields bit for bit, mixed within 1e-5 of exact."""
    c = make("stretch")
    ref, cnt = run_oracle(oracle, c, counters=True)
    assert cnt["tets"] > 6 * 12 ** 3  # the criterion refined something
    out, _, _ = run_psi(gpu, c, precision="fp64")
    assert gpu.last_stats()["tets"] == cnt["tets"]
    for f in ref:
        assert np.array_equal(out[f], ref[f]), f
    out, _, _ = run_psi(gpu, c, precision="mixed")
    ex = run_oracle(oracle, c, kind="exact")
    check_vs_exact_and_reference(out, ref, ex, MIXED_TOL, "stretch")
    assert mass_error(out["m"], total_mass(c)) <= MASS_TOL


def test_mixed_accumulates_into_existing_grid(gpu, oracle):
    """The mixed path merges each voxel's new fragments into the fields already
    on the grid in one step; the result is the reference's sequential update
    within the mixed bound."""
    a, b = make("c2_small"), make("c2_order1")
    b["fields"] = a["fields"]
    ref = run_oracle(oracle, a)
    ref = oracle.voxelize("restatement", n=b["n"], bounds=b["bounds"], pos=b["pos"].reshape(-1, 3),
                          vel=b["vel"].reshape(-1, 3), conn=oracle.block_connectivity((16, 16, 16), True),
                          periodic_box=b["periodic_box"], fields=b["fields"], out=ref)
    _, grid, _ = run_psi(gpu, a, precision="mixed")
    out, _, _ = run_psi(gpu, b, grid=grid, precision="mixed")
    check(field_errors(out, ref), MIXED_TOL, "accumulate mixed")


def test_chunked_streaming_matches(gpu, oracle, monkeypatch):
    """Tets streamed in element chunks (a tiny item budget) give the same result."""
    ref, _ = reference(oracle, "c2_small")
    monkeypatch.setenv("PSIB_ITEM_BUDGET", "5000")
    out, _, _ = run_psi(gpu, make("c2_small"))
    assert gpu.last_stats()["chunks"] > 5
    check(field_errors(out, ref), FP64_TOL, "chunked")
    out, _, _ = run_psi(gpu, make("c2_small"), deterministic=True)
    for f in ref:
        assert np.array_equal(out[f], ref[f]), f


def test_tutorial_plane_wave_mass(gpu):
    """The tutorial's plane-wave block mesh, 64^3 particles onto 64^3, lvl 2,
    tol 0.05 (Tutorial.ipynb cell 12; printed global error 0.0)."""
    nside = 64
    g = np.mgrid[:nside, :nside, :nside]
    pos = (np.rollaxis(g, 0, 4).copy() + 0.5) / nside
    pos[..., 0] += 0.1 * np.sin(2 * np.pi * pos[..., 0])
    pos[..., 1] += 0.005 * np.sin(6 * np.pi * pos[..., 1])
    pos[..., 2] += 0.002 * np.sin(8 * np.pi * pos[..., 2])
    box = (3 * (0.0,), 3 * (1.0,))
    mesh = gpu.Mesh(loader="block", pos=pos, periodic_box=box)
    for prec in ("fp64", "mixed"):
        grid = gpu.Grid(n=(64, 64, 64), bounds=box)
        gpu.voxels(grid=grid, mesh=mesh, refine_tolerance=0.05, refine_max_lvl=2, precision=prec)
        assert mass_error(grid.fields["m"], np.sum(mesh.mass)) <= MASS_TOL


def test_full_size_properties(gpu):
    """128^3 particles, rms 2 cells, onto 256^3 with all order-2 fields: mass
    conserved to 1e-13 in every precision; mixed within 1e-5 of the FP64-central
    result, and of the FP64 (reference) result within 1e-5 plus the distance
    between the two FP64 results."""
    from pypsi_b200.synth import zeldovich

    pos, vel = zeldovich(128, 2.0, 2024)
    box = ((0.0,) * 3, (100.0,) * 3)
    mesh = gpu.Mesh(loader="block", pos=pos, vel=vel, periodic_box=box)
    fields = ["x", "v", "xx", "xv", "vv"]
    outs = {}
    for prec in ("fp64", "mixed", "fp64-central"):
        grid = gpu.Grid(n=(256, 256, 256), bounds=box, fields=fields)
        gpu.voxels(grid=grid, mesh=mesh, precision=prec)
        assert mass_error(grid.fields["m"], 128 ** 3) <= MASS_TOL, prec
        outs[prec] = {k: np.array(v) for k, v in grid.fields.items()}
        del grid
    check_vs_exact_and_reference(outs["mixed"], outs["fp64"], outs["fp64-central"], MIXED_TOL, "full")


def test_32cube_to_64cube_density_bitwise_against_compiled_reference(gpu, oracle):
    """The reference's CPU-runnable workload at its own size: 32^3 particles
    (rms 0.3 cells) onto a 64^3 grid, density only, against the reference's C
    code compiled from its sources -- bit for bit in FP64, 1e-5 in mixed."""
    from pypsi_b200.synth import zeldovich

    pos, vel = zeldovich(32, 0.3, 2031)
    c = {"kind": "block", "pos": pos, "vel": vel, "mass": None, "periodic_box": ((0.0,) * 3, (100.0,) * 3),
         "n": (64, 64, 64), "bounds": ((0.0,) * 3, (100.0,) * 3), "fields": [], "reftol": 1.0, "maxlvl": 0}
    kind = "reference" if oracle.available("reference") else "restatement"
    ref = run_oracle(oracle, c, kind=kind)
    out, _, _ = run_psi(gpu, c, precision="fp64")
    assert np.array_equal(out["m"], ref["m"])
    out, _, _ = run_psi(gpu, c, precision="mixed")
    check(field_errors(out, ref), MIXED_TOL, "32^3 -> 64^3")
    assert mass_error(out["m"], 32 ** 3) <= MASS_TOL


@pytest.mark.parametrize("name", NAMES)
def test_fp64_breadth_first_equals_depth_first(gpu, name, monkeypatch):
    """The FP64 walk runs breadth first (the mixed walk's level launches, FP64 positions and q);
    its fields, fragments and splits equal the depth-first FP64 kernel's bit for bit."""
    c = make(name)
    monkeypatch.setenv("PSIB_BFS64", "0")
    want, _, _ = run_psi(gpu, c, precision="fp64")
    st0 = gpu.last_stats()
    assert st0["walk_bytes"] == 0
    monkeypatch.setenv("PSIB_BFS64", "1")
    got, _, _ = run_psi(gpu, c, precision="fp64")
    st1 = gpu.last_stats()
    if name != "big_tet":  # a tree deeper than the walk's levels goes to the depth-first kernel
        assert st1["walk_bytes"] > 0
    for f in want:
        assert np.array_equal(got[f], want[f]), (name, f, np.abs(got[f] - want[f]).max())
    assert st1["fragments"] == st0["fragments"]
    assert st1["splits"] == st0["splits"]


def test_fp64_breadth_first_many_passes(gpu, monkeypatch):
    """64^3 particles (rms 2 cells) onto 128^3 with every field, the walk's queues held to
    2^18 box voxels so that it takes many passes, and in element chunks: bit for bit the
    depth-first FP64 kernel, and the mass to 1e-13."""
    from pypsi_b200.synth import zeldovich

    pos, vel = zeldovich(64, 2.0, 2042, box=50.0)
    c = {"kind": "block", "pos": pos, "vel": vel, "mass": None, "periodic_box": ((0.0,) * 3, (50.0,) * 3),
         "n": (128, 128, 128), "bounds": ((0.0,) * 3, (50.0,) * 3), "fields": ["x", "v", "xx", "xv", "vv"],
         "reftol": 1.0, "maxlvl": 0}
    monkeypatch.setenv("PSIB_BFS64", "0")
    want, _, _ = run_psi(gpu, c, precision="fp64")
    monkeypatch.setenv("PSIB_BFS64", "1")
    monkeypatch.setenv("PSIB_BFS_CAP", str(1 << 18))
    monkeypatch.setenv("PSIB_ITEM_BUDGET", str(400000))
    got, _, _ = run_psi(gpu, c, precision="fp64")
    assert gpu.last_stats()["chunks"] > 1
    for f in want:
        assert np.array_equal(got[f], want[f]), (f, np.abs(got[f] - want[f]).max())
    assert mass_error(got["m"], 64 ** 3) <= MASS_TOL
