"""PSI.Mesh(loader='gadget2' | 'gevolution'): snapshot files read into the
periodic trilinear mesh of src/mesh.c:35-302 / src/PSI.c:659-709.

The loaders are host code; these tests need no GPU.  Each synthetic snapshot
is read three ways -- the PSI module (psib_load_*), the oracle's numpy
restatement and the reference's own compiled load_gadget2 / load_gevolution --
and all three must agree bit for bit.  A deposit from a loaded snapshot is in
test_gpu_loaders.py."""
import ctypes
import os

import numpy as np
import pytest

from snapshots import make_snapshot, write_snapshot

REF_SNAPSHOT = "/root/reference/tutorial/snapshot_010"


def mesh_arrays(mesh):
    return mesh.pos, mesh.vel, mesh.mass, mesh.connectivity


def check_same(a, b):
    for x, y, name in zip(a, b, ("pos", "vel", "mass", "connectivity")):
        assert x.shape == y.shape and x.dtype == y.dtype, name
        assert np.array_equal(x, y), name


@pytest.mark.parametrize("flavour,n", [("gadget2", 6), ("gadget2", 8), ("gevolution", 8), ("gevolution", 12)])
def test_synthetic_snapshot_matches_restatement_and_reference(psi, oracle, tmp_path, flavour, n):
    path = str(tmp_path / "snap")
    pos, vel = make_snapshot(path, n, flavour=flavour, seed=n)
    mesh = psi.Mesh(loader=flavour, filename=path)
    got = mesh_arrays(mesh)
    assert mesh.wrapbox == ((0.0, 0.0, 0.0), (40.0, 40.0, 40.0))
    assert got[0].shape == (n ** 3, 3) and got[3].shape == (n ** 3, 8) and got[2].shape == (n ** 3,)
    # the particles are back in ID order, widened from float32
    assert np.array_equal(got[0], pos.astype(np.float32).astype(np.float64))
    assert np.array_equal(got[1], vel.astype(np.float32).astype(np.float64))
    assert np.all(got[2] == 15.0 / n ** 3)
    rp, rv, rm, rc, rbox = oracle.load_snapshot("restatement", path, flavour)
    assert rbox == 40.0
    check_same(got, (rp, rv, rm, rc))
    if oracle.available("reference"):
        fp, fv, fm, fc, fbox = oracle.load_snapshot("reference", path, flavour)
        assert fbox == 40.0
        check_same(got, (fp, fv, fm, fc))


@pytest.mark.parametrize("n", [4, 8])
def test_gevolution_elements_are_lattice_cubes(psi, tmp_path, n):
    """Every gevolution element joins the 8 corners of one lattice cell, in the
    corner order 4*ii + 2*jj + kk, and the elements tile the periodic lattice."""
    from snapshots import gevolution_rows

    path = str(tmp_path / "snap")
    make_snapshot(path, n, flavour="gevolution")
    conn = psi.Mesh(loader="gevolution", filename=path).connectivity
    rows = gevolution_rows(n)
    ijk = np.stack([rows // (n * n), (rows // n) % n, rows % n], axis=1)
    base = ijk[conn[:, 0]]
    for c in range(8):
        off = np.array([(c >> 2) & 1, (c >> 1) & 1, c & 1])
        assert np.array_equal(ijk[conn[:, c]], (base + off) % n)
    cells = (base[:, 0] * n + base[:, 1]) * n + base[:, 2]
    assert np.array_equal(np.sort(cells), np.arange(n ** 3))


def test_c_abi_peek_and_load(tmp_path):
    import pypsi_b200

    lib = pypsi_b200.lib
    path = str(tmp_path / "snap")
    make_snapshot(path, 4, box=12.5, mass1=3.0)
    np_, box = ctypes.c_longlong(), ctypes.c_double()
    assert lib.psib_peek_gadget2(path.encode(), ctypes.byref(np_), ctypes.byref(box)) == 0
    assert np_.value == 64 and box.value == 12.5
    pos, vel, mass = np.zeros((64, 3)), np.zeros((64, 3)), np.zeros(64)
    conn = np.zeros((64, 8), np.int32)
    dp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    lib.psib_load_gadget2.argtypes = [ctypes.c_char_p, ctypes.c_longlong] + [ctypes.c_void_p] * 4
    assert lib.psib_load_gadget2(path.encode(), 64, dp(pos), dp(vel), dp(mass), dp(conn)) == 0
    assert np.all(mass == 3.0 / 64)
    # a capacity that disagrees with the header is an argument error
    assert lib.psib_load_gadget2(path.encode(), 63, dp(pos), dp(vel), dp(mass), dp(conn)) == 1
    lib.psib_last_error.restype = ctypes.c_char_p
    assert b"hold 63 particles" in lib.psib_last_error()


def test_bad_files(psi, tmp_path):
    with pytest.raises(ValueError, match="Bad file name"):
        psi.Mesh(loader="gadget2", filename=str(tmp_path / "missing"))
    with pytest.raises(ValueError, match="Bad file name"):
        psi.Mesh(loader="gadget2")
    from snapshots import lattice_particles

    pos, vel = lattice_particles(4, 10.0)
    # IDs counted from 1, as many Gadget initial conditions number them
    p = str(tmp_path / "from1")
    write_snapshot(p, pos, vel, 1.0, 10.0, ids=np.arange(1, 65))
    with pytest.raises(ValueError, match="Could not read .*outside"):
        psi.Mesh(loader="gadget2", filename=p)
    p = str(tmp_path / "repeat")
    write_snapshot(p, pos, vel, 1.0, 10.0, ids=np.r_[np.arange(63), 0])
    with pytest.raises(ValueError, match="Could not read .*repeated"):
        psi.Mesh(loader="gadget2", filename=p)
    # 60 particles are not a cubic lattice
    p = str(tmp_path / "ragged")
    write_snapshot(p, pos[:60], vel[:60], 1.0, 10.0, ids=np.arange(60))
    with pytest.raises(ValueError, match="cubic lattice"):
        psi.Mesh(loader="gadget2", filename=p)
    # gevolution tiles need a side that is a multiple of 4
    p = str(tmp_path / "gev6")
    make_snapshot(p, 6, flavour="gadget2")
    with pytest.raises(ValueError, match="multiple of 4"):
        psi.Mesh(loader="gevolution", filename=p)
    # a truncated file
    p = str(tmp_path / "short")
    make_snapshot(p, 4)
    raw = open(p, "rb").read()
    open(p, "wb").write(raw[:-100])
    with pytest.raises(ValueError, match="Could not read"):
        psi.Mesh(loader="gadget2", filename=p)
    # a header that claims more particles than the blocks hold
    p = str(tmp_path / "lying")
    write_snapshot(p, pos, vel, 1.0, 10.0, header_npart=125)
    with pytest.raises(ValueError, match="Could not read"):
        psi.Mesh(loader="gadget2", filename=p)


def test_empty_snapshot(psi, tmp_path):
    p = str(tmp_path / "empty")
    write_snapshot(p, np.zeros((0, 3)), np.zeros((0, 3)), 1.0, 5.0)
    mesh = psi.Mesh(loader="gadget2", filename=p)
    assert mesh.pos.shape == (0, 3) and mesh.connectivity.shape == (0, 8)
    assert mesh.wrapbox == ((0.0, 0.0, 0.0), (5.0, 5.0, 5.0))


@pytest.mark.skipif(not os.path.exists(REF_SNAPSHOT), reason="the reference's tutorial snapshot is not present")
def test_tutorial_snapshot_matches_reference(psi, oracle):
    """The snapshot the reference's tutorial loads (32^3 particles, box 40)."""
    mesh = psi.Mesh(loader="gadget2", filename=REF_SNAPSHOT)
    assert mesh.pos.shape == (32768, 3)
    assert mesh.wrapbox == ((0.0, 0.0, 0.0), (40.0, 40.0, 40.0))
    check_same(mesh_arrays(mesh), oracle.load_snapshot("restatement", REF_SNAPSHOT)[:4])
    if oracle.available("reference"):
        check_same(mesh_arrays(mesh), oracle.load_snapshot("reference", REF_SNAPSHOT)[:4])
