"""The density deposit that allocates nothing (psib_voxels_density_noalloc).

It exists for callers that must not have the library allocate device memory,
such as an application whose own pool allocator owns all of the GPU's memory,
or a time-critical loop that cannot afford an allocation's synchronisation.
Here it is called through the C ABI on tets held in device memory, twice in a
row, and each result is checked against psib_voxels on the same tets (simplex
elements) at the FP64 parity tolerance.  A tet too large for its fixed scratch
must be rejected with a clear error.  This file is collected last on purpose.
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


def test_noalloc_matches_psib_voxels_twice(gpu):
    import torch

    from pypsi_b200 import capi

    f = _entry()
    pos, mass = _tets()
    nt = len(mass)
    n, bounds = (24, 24, 24), ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
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


def test_noalloc_rejects_tet_beyond_its_scratch(gpu):
    import torch

    from pypsi_b200 import capi

    f = _entry()
    big = np.array([[[0.01, 0.02, 0.03], [0.98, 0.05, 0.04], [0.03, 0.97, 0.06], [0.05, 0.04, 0.99]]])
    dpos = torch.from_numpy(big.reshape(-1, 3)).cuda()
    m = torch.zeros((64, 64, 64), dtype=torch.float64, device="cuda")
    g = capi.make_grid((64, 64, 64), ((0.0,) * 3, (1.0,) * 3), {"m": m.data_ptr()})
    rc = f(ctypes.byref(g), dpos.data_ptr(), None, 1, None)
    assert rc == 1  # PSIB_ERR_ARG
    assert b"too large" in capi.lib.psib_last_error()
    assert not m.any()
