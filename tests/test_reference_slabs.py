"""The reference arm of bench.py splits the 256^3 grid into window slabs along
x, one process each, every process running the reference's psi_voxels over
the whole periodic mesh on its slab.  These checks (CPU only, the compiled
reference) show that the slabs together are the whole deposit: each voxel's
mass equals the single full-window call's to rounding, periodic images at the
box faces included, and that the arm maps none of this library's native code.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
from pypsi_b200.synth import zeldovich

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BOX = ((0.0,) * 3, (100.0,) * 3)
FIELDS = ["x", "v", "xx", "xv", "vv"]


def _slabs(n_grid, nslabs):
    d = 100.0 / n_grid
    for s in range(nslabs):
        i0, i1 = n_grid * s // nslabs, n_grid * (s + 1) // nslabs
        yield i0, i1, ((i0 * d, 0.0, 0.0), (i1 * d, 100.0, 100.0))


@pytest.mark.skipif(not O.available("reference"), reason="the compiled reference is absent")
@pytest.mark.parametrize("nslabs", [3, 4])
def test_window_slabs_are_the_whole_deposit(nslabs):
    n, ng = 12, 24
    pos, vel = zeldovich(n, 2.0, 1234)
    pos, vel = pos.reshape(-1, 3), vel.reshape(-1, 3)
    conn = O.block_connectivity((n,) * 3, True)
    full = O.voxelize("reference", n=(ng,) * 3, bounds=BOX, pos=pos, vel=vel, conn=conn, periodic_box=BOX,
                      fields=FIELDS)
    parts = [O.voxelize("reference", n=(i1 - i0, ng, ng), bounds=b, pos=pos, vel=vel, conn=conn, periodic_box=BOX,
                        fields=FIELDS) for i0, i1, b in _slabs(ng, nslabs)]
    union = {f: np.concatenate([p[f] for p in parts], axis=0) for f in full}
    # mass per voxel: the same fragments, cut in another order at the slab faces
    m, mu = full["m"], union["m"]
    assert np.all((m > 0) == (mu > 0))
    assert np.max(np.abs(mu - m)) <= 1e-12 * np.max(m)
    assert abs(mu.sum() - n ** 3) <= 1e-13 * n ** 3
    # first moments are well conditioned in the reference's arithmetic
    live = m > 0
    for f in ("x", "v"):
        scale = np.max(np.abs(full[f][live]))
        assert np.max(np.abs(union[f][live] - full[f][live])) <= 1e-10 * scale, f


def test_reference_arm_maps_no_library_code():
    """The reference arm's inputs come from pure-numpy helpers: importing them
    maps neither libpsi_b200.so nor the PSI extension."""
    code = (
        "import sys; sys.path[:0] = [%r, %r]\n"
        "import bench\n"
        "bench._ref_inputs()\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libpsi_b200' not in maps and 'PSI.cpython' not in maps, 'library code mapped'\n"
        "print('ok')\n" % (ROOT, os.path.join(ROOT, "oracle")))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr
