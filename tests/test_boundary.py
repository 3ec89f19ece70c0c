"""The drop-in boundary on a machine without a GPU: the C ABI library loads and
exports every entry point include/psi_b200.h declares, and the PSI module's
Grid / Mesh / voxels validate arguments as src/PSI.c does.  No GPU compute."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "psi_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(psib_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import pypsi_b200

    lib = ctypes.CDLL(pypsi_b200.LIB_PATH)
    syms = declared_symbols()
    assert "psib_voxels" in syms
    for s in syms:
        assert hasattr(lib, s), s


def test_abi_version_and_no_device_error(psi):
    import pypsi_b200

    lib = pypsi_b200.lib
    assert lib.psib_abi_version() == 2
    lib.psib_voxels.restype = ctypes.c_int
    # argument validation runs before any device work
    assert lib.psib_voxels(None, None, 0, ctypes.c_double(1.0), 0, None) == 1  # PSIB_ERR_ARG
    lib.psib_last_error.restype = ctypes.c_char_p
    assert b"required" in lib.psib_last_error()


def test_grid_defaults(psi):
    g = psi.Grid()
    assert g.type == "cart"
    assert g.n == (32, 32, 32)
    assert g.bounds == ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    assert g.d == (1 / 32, 1 / 32, 1 / 32)
    assert list(g.fields) == ["m"] and g.fields["m"].shape == (32, 32, 32)
    assert g.fields["m"].dtype == np.float64 and not g.fields["m"].any()


def test_grid_fields_and_shapes(psi):
    g = psi.Grid(n=(3, 4, 5), bounds=((0, 1, 2), (3, 5, 7)), fields=["x", "v", "xx", "vx", "vv"])
    assert g.d == (1.0, 1.0, 1.0)
    assert g.fields["x"].shape == (3, 4, 5, 3)
    assert g.fields["xv"].shape == (3, 4, 5, 3, 3)
    assert sorted(g.fields) == ["m", "v", "vv", "x", "xv", "xx"]


@pytest.mark.parametrize("kw,exc,msg", [
    (dict(type="sphere"), ValueError, "Invalid grid type: sphere"),
    (dict(type="hpring"), ValueError, "Grid type hpring is not yet implemented"),
    (dict(n=(1, 2)), TypeError, "n must be a tuple containing 3 integers"),
    (dict(bounds=((0, 0), (1, 1))), TypeError, "bounds must be a tuple containing two tuples of 3 values each"),
    (dict(fields=["q"]), ValueError, "Unrecognized field identifier: q"),
    (dict(fields=[1]), TypeError, "Field identifiers must be strings"),
    (dict(fields=["xx"]), ValueError, "Field 'xx' requires you to also provide field 'x'."),
    (dict(fields=["x", "xv"]), ValueError, "Field 'xv' requires you to also provide fields 'x' and 'v'."),
    (dict(fields=["vv"]), ValueError, "Field 'vv' requires you to also provide field 'v'."),
])
def test_grid_errors(psi, kw, exc, msg):
    with pytest.raises(exc, match=re.escape(msg)):
        psi.Grid(**kw)


def test_block_mesh_matches_reference_connectivity(psi, oracle):
    pos = np.random.default_rng(0).random((3, 4, 5, 3))
    for box in (None, ((0, 0, 0), (1, 1, 1))):
        kw = dict(loader="block", pos=pos)
        if box:
            kw["periodic_box"] = box
        m = psi.Mesh(**kw)
        exp = oracle.block_connectivity((3, 4, 5), box is not None)
        assert np.array_equal(m.connectivity, exp)
        assert m.mass.shape == ((3, 4, 5) if box else (2, 3, 4))
        assert np.all(m.mass == 1.0) and not m.vel.any()
        assert m.wrapbox == (((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)) if box else None)


@pytest.mark.parametrize("kw,exc,msg", [
    (dict(loader="array", pos=[[0.0, 0, 0]], connectivity=np.zeros((1, 4), np.int32)), TypeError,
     "pos must be a numpy array"),
    (dict(loader="array", pos=np.zeros((4, 3), np.float32), connectivity=np.zeros((1, 4), np.int32)), TypeError,
     "pos must be an array of doubles"),
    (dict(loader="array", pos=np.zeros((4, 2)), connectivity=np.zeros((1, 4), np.int32)), TypeError,
     "pos must be a 2D array with shape (npart, 3)"),
    (dict(loader="array", pos=np.zeros((4, 3)), connectivity=np.zeros((1, 4), np.int64)), TypeError,
     "connectivity must be an array of ints"),
    (dict(loader="array", pos=np.zeros((4, 3)), connectivity=np.zeros((1, 5), np.int32)), TypeError,
     "nverts_per_elem is 4, 8, or 27"),
    (dict(loader="array", pos=np.zeros((4, 3)), connectivity=np.zeros((1, 4), np.int32), vel=np.zeros((3, 3))),
     TypeError, "if provided, vel must have the same shape as pos"),
    (dict(loader="array", pos=np.zeros((4, 3)), connectivity=np.zeros((1, 4), np.int32), mass=np.zeros(2)),
     TypeError, "if provided, mass must be a 1D array of length nelem"),
    (dict(loader="block", pos=np.zeros((2, 2, 2))), TypeError, "pos must be a 4D array with shape (nx, ny, nz, 3)"),
    (dict(loader="block", pos=np.zeros((2, 2, 2, 3)), mass=np.ones((2, 2, 2))), TypeError,
     "if provided, mass must be a 3D array of shape (nelemx, nelemy, nelemz)"),
    (dict(loader="block", pos=np.zeros((2, 2, 2, 3)), periodic_box=(0, 1)), TypeError,
     "periodic_box must be a tuple containing two tuples of 3 values each"),
    (dict(loader="nbody"), ValueError, "Invalid mesh loader."),
])
def test_mesh_errors(psi, kw, exc, msg):
    with pytest.raises(exc, match=re.escape(msg)):
        psi.Mesh(**kw)


def test_voxels_argument_errors(psi):
    g = psi.Grid(n=(4, 4, 4))
    m = psi.Mesh(loader="block", pos=np.random.default_rng(1).random((3, 3, 3, 3)))
    with pytest.raises(ValueError, match="Invalid mode for PSI.voxels\\(\\): fast"):
        psi.voxels(g, m, mode="fast")
    with pytest.raises(ValueError, match="Invalid precision"):
        psi.voxels(g, m, precision="fp16")
    with pytest.raises(TypeError):
        psi.voxels(g, "not a mesh")


def test_voxels_fails_loudly_without_gpu(psi):
    if psi.device_count() > 0:
        pytest.skip("a GPU is present")
    g = psi.Grid(n=(4, 4, 4))
    m = psi.Mesh(loader="block", pos=np.random.default_rng(1).random((3, 3, 3, 3)))
    with pytest.raises(RuntimeError, match="no CUDA device"):
        psi.voxels(g, m)
    assert not g.fields["m"].any()


def test_query_and_vdf_argument_errors(psi):
    """PSI.RStarTree / PSI.VDF keep the reference's argument checks
    (src/PSI.c:817-835, :865-876, :1022-1040); the C entry points reject
    missing arrays before any device work."""
    import ctypes

    import pypsi_b200

    m = psi.Mesh(loader="block", pos=np.random.default_rng(1).random((3, 3, 3, 3)))
    with pytest.raises(TypeError):
        psi.RStarTree("not a mesh")
    with pytest.raises(TypeError):
        psi.VDF(m, (0.5, 0.5))
    with pytest.raises(TypeError):
        psi.VDF(m, (0.5, 0.5, 0.5), tree="not a tree")
    tree = psi.RStarTree(m)
    assert tree.mesh is m
    with pytest.raises(TypeError, match="two tuples of 3 values"):
        tree.query(((0, 0), (1, 1)))
    lib = pypsi_b200.lib
    lib.psib_last_error.restype = ctypes.c_char_p
    off = (ctypes.c_longlong * 2)()
    assert lib.psib_query_elements(None, None, None, ctypes.c_longlong(1), off, None, ctypes.c_longlong(0), None) == 1
    assert b"window" in lib.psib_last_error()
    assert lib.psib_sample_vdf(None, None, None, ctypes.c_longlong(1), ctypes.c_double(1.0), 0, off, None, None,
                               ctypes.c_longlong(0), None) == 1
    assert b"window" in lib.psib_last_error()


def test_query_and_vdf_fail_loudly_without_gpu(psi):
    if psi.device_count() > 0:
        pytest.skip("a GPU is present")
    m = psi.Mesh(loader="block", pos=np.random.default_rng(1).random((3, 3, 3, 3)), periodic_box=((0, 0, 0), (1, 1, 1)))
    with pytest.raises(RuntimeError, match="no CUDA device"):
        psi.VDF(m, (0.5, 0.5, 0.5))
    with pytest.raises(RuntimeError, match="no CUDA device"):
        psi.RStarTree(m).query(((0, 0, 0), (1, 1, 1)))
    g = psi.Grid(n=(4, 4, 4))
    with pytest.raises(RuntimeError, match="no CUDA device"):
        psi.voxels(g, m, mode="annihilation")


def test_ctypes_wrappers_fail_loudly_without_gpu(psi):
    """The device-array wrappers raise the library's error; nothing falls back to the CPU."""
    if psi.device_count() > 0:
        pytest.skip("a GPU is present")
    from pypsi_b200 import capi

    pos = np.random.default_rng(1).random((27, 3))
    with pytest.raises(capi.PsibError, match="no CUDA device"):
        capi.sample_vdf(np.zeros((4, 3)), pos, block_dims=(3, 3, 3), periodic_box=((0, 0, 0), (1, 1, 1)))
    assert capi.tree_window(None) == ((-1.0e30,) * 3, (1.0e30,) * 3)
    assert capi.tree_window(((0, 0, 0), (2, 3, 4))) == ((0.0, 0.0, 0.0), (2.0, 3.0, 4.0))
