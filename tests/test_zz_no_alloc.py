"""The density deposit that allocates nothing (psib_voxels_density_noalloc).

It exists for callers that must not have the library allocate device memory,
such as an application whose own pool allocator owns all of the GPU's memory,
or a time-critical loop that cannot afford an allocation's synchronisation.
Here it is called through the C ABI on tets held in device memory, twice in a
row, and each result is checked against psib_voxels on the same tets (simplex
elements) at the FP64 parity tolerance, also for tets that cross the faces of
the grid window and at the depth limit (16x16x16 voxels, 12 levels).  A call
with a tet too large for the fixed scratch (16x16x32, 13 levels) must fail
with a clear error and leave m untouched, even when its other tets are small.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from pypsi_b200.metrics import field_errors

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _entry():
    from pypsi_b200 import capi, lib

    f = lib.psib_voxels_density_noalloc
    f.argtypes = [ctypes.POINTER(capi.Grid), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _tets(seed=31, nt=500):
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.15, 0.85, (nt, 1, 3))
    pos = np.clip(c + rng.normal(0.0, 0.05, (nt, 4, 3)), 0.001, 0.999)
    return pos, rng.uniform(0.5, 1.5, nt)


def _window_tets(seed=32, nt=400):
    """Tets that cross the faces, edges and corners of the window [0,1]^3, and
    one wholly outside it."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.05, 1.05, (nt, 1, 3))
    pos = c + rng.normal(0.0, 0.06, (nt, 4, 3))
    pos[0] = np.array([[1.2, 1.2, 1.2], [1.3, 1.2, 1.2], [1.2, 1.3, 1.2], [1.2, 1.2, 1.3]])
    return pos, rng.uniform(0.5, 1.5, nt)


def _depth_tet(nx, ny, nz, d):
    """A tet whose voxel index box is nx x ny x nz voxels of size d from the origin."""
    lo, hx, hy, hz = 0.5 * d, (nx - 0.5) * d, (ny - 0.5) * d, (nz - 0.5) * d
    return np.array([[[lo, lo, lo], [hx, lo, lo], [lo, hy, lo], [lo, lo, hz]]])


def _compare_twice(pos, mass, n, bounds):
    """Two calls of the entry point in a row, each against psib_voxels."""
    import torch

    from pypsi_b200 import capi

    f = _entry()
    nt = len(mass)
    dpos = torch.from_numpy(pos.reshape(-1, 3)).cuda()
    dmass = torch.from_numpy(mass).cuda()
    conn = torch.arange(4 * nt, dtype=torch.int32, device="cuda").reshape(nt, 4)

    ref = torch.zeros(n, dtype=torch.float64, device="cuda")
    capi.voxels_device({"m": ref}, n, bounds, dpos, None, dmass, connectivity=conn)
    ref_np = ref.cpu().numpy()
    assert ref_np.sum() > 0.5 * mass.sum()

    stream = torch.cuda.current_stream()
    for call in range(2):
        m = torch.zeros(n, dtype=torch.float64, device="cuda")
        g = capi.make_grid(n, bounds, {"m": m.data_ptr()})
        rc = f(ctypes.byref(g), dpos.data_ptr(), dmass.data_ptr(), nt, ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, (call, capi.lib.psib_last_error())
        errs = field_errors({"m": m.cpu().numpy()}, {"m": ref_np})
        assert errs["m"]["rel"] <= FP64_TOL and errs["dead_m"] == 0.0, (call, errs)


def test_noalloc_matches_psib_voxels_twice(gpu):
    pos, mass = _tets()
    _compare_twice(pos, mass, (24, 24, 24), ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)))


def test_noalloc_window_clip_matches_psib_voxels(gpu):
    pos, mass = _window_tets()
    _compare_twice(pos, mass, (20, 24, 28), ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)))


@pytest.mark.parametrize("shape", ["16x16x16", "4096x1x1"])
def test_noalloc_depth_limit_accepted(gpu, shape):
    """Index boxes whose bisection is exactly 12 levels deep: 4 + 4 + 4 and 12 + 0 + 0."""
    if shape == "16x16x16":
        d = 1.0 / 64
        n = (64, 64, 64)
        pos = np.concatenate([_depth_tet(16, 16, 16, d), _depth_tet(16, 16, 16, d) + 20 * d])
    else:
        n = (4096, 4, 4)
        dx = 1.0 / 4096
        pos = np.array([[[0.5 * dx, 0.02, 0.02], [4095.5 * dx, 0.03, 0.04], [0.4, 0.23, 0.05],
                         [0.7, 0.04, 0.22]]])
        pos = np.concatenate([pos, pos + [0.0, 0.5, 0.25]])
    _compare_twice(pos, np.array([1.0, 2.0]), n, ((0.0,) * 3, (1.0,) * 3))


@pytest.mark.parametrize("which", ["alone", "among_small_tets"])
def test_noalloc_rejects_tet_beyond_its_scratch(gpu, which):
    import torch

    from pypsi_b200 import capi

    f = _entry()
    d = 1.0 / 64
    big = _depth_tet(16, 16, 32, d)  # 4 + 4 + 5 = 13 levels
    if which == "among_small_tets":
        small, _ = _tets(seed=33, nt=300)
        big = np.concatenate([small[:150], big, small[150:]])
    dpos = torch.from_numpy(np.ascontiguousarray(big.reshape(-1, 3))).cuda()
    m = torch.full((64, 64, 64), 0.25, dtype=torch.float64, device="cuda")
    g = capi.make_grid((64, 64, 64), ((0.0,) * 3, (1.0,) * 3), {"m": m.data_ptr()})
    rc = f(ctypes.byref(g), dpos.data_ptr(), None, len(big), None)
    assert rc == 1  # PSIB_ERR_ARG
    assert b"too large" in capi.lib.psib_last_error()
    assert bool((m == 0.25).all()), "a rejected call must deposit nothing"
