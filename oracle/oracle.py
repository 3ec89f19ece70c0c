"""ctypes front end of the test oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline / reference legs as the checker.  The product package
``pypsi_b200`` never imports it.

Two back ends with one interface:

* ``restatement`` -- ``_build/liboracle.so`` from ``psi_oracle.c``, a step by
  step C restatement of the reference density path with work counters;
* ``exact``       -- ``_build/liboracle_exact.so``, the same restatement with
  quad-precision (__float128) arithmetic: the result the reference's algorithm
  computes without rounding, to measure the reference's own rounding error;
* ``reference``   -- ``_ref/libpsiref.so``, the reference's own sources
  (src/cpsi.c, src/geometry.c, src/refine.c, ...) compiled unchanged; its entry
  ``psi_voxels`` is declared at src/PSI.c:39 and defined at src/cpsi.c:41.

``voxelize`` returns the grid fields in the reference's layout
(src/PSI.c:124-186): ``m`` (nx,ny,nz), ``x``/``v`` (...,3), ``xx``/``xv``/``vv``
(...,3,3), all float64.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "_build", "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libpsiref.so")
LIB_EXACT = os.path.join(HERE, "_build", "liboracle_exact.so")
_PATHS = {"restatement": LIB_ORACLE, "exact": LIB_EXACT, "reference": LIB_REF}
FIELD_NAMES = ("m", "x", "v", "xx", "xv", "vv")


def build(ref_root: str = "/root/reference", quiet: bool = True) -> None:
    """Compile the restatement, and the reference when its tree is present."""
    targets = ["oracle"]
    if os.path.isdir(os.path.join(ref_root, "src")):
        targets.append("ref")
    out = subprocess.run(["make", "-C", HERE, f"REF={ref_root}", *targets],
                         capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


# ---- restatement structs (psi_oracle.c) ----
class _OgGrid(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("win", (C.c_double * 3) * 2), ("d", C.c_double * 3),
                ("f", C.POINTER(C.c_double) * 6)]


class _OgMesh(C.Structure):
    _fields_ = [("elemtype", C.c_int), ("npart", C.c_int), ("nelem", C.c_int),
                ("pos", C.POINTER(C.c_double)), ("vel", C.POINTER(C.c_double)),
                ("mass", C.POINTER(C.c_double)), ("conn", C.POINTER(C.c_int)),
                ("periodic", C.c_int), ("box", (C.c_double * 3) * 2)]


class Counters(C.Structure):
    _fields_ = [("elements_kept", C.c_longlong), ("tets", C.c_longlong),
                ("tet_images", C.c_longlong), ("fragments", C.c_longlong),
                ("splits", C.c_longlong), ("frag_verts", C.c_longlong),
                ("max_verts", C.c_longlong), ("errors", C.c_longlong)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


# ---- reference structs (include/grid.h:46-53, include/mesh.h:42-52) ----
class _PsiGrid(C.Structure):
    _fields_ = [("type", C.c_int), ("dim", C.c_int), ("fields", C.POINTER(C.c_double) * 16),
                ("window", (C.c_double * 3) * 2), ("n", C.c_int * 3), ("d", C.c_double * 3)]


class _PsiMesh(C.Structure):
    _fields_ = [("elemtype", C.c_int), ("dim", C.c_int), ("pos", C.POINTER(C.c_double)),
                ("vel", C.POINTER(C.c_double)), ("mass", C.POINTER(C.c_double)),
                ("npart", C.c_int), ("nelem", C.c_int), ("connectivity", C.POINTER(C.c_int)),
                ("box", (C.c_double * 3) * 2), ("periodic", C.c_int)]


_libs: dict[str, C.CDLL] = {}


def _lib(kind: str) -> C.CDLL:
    if kind not in _libs:
        path = _PATHS[kind]
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (run oracle.build())")
        lib = C.CDLL(path)
        if kind != "reference":
            lib.oracle_voxels.argtypes = [C.POINTER(_OgGrid), C.POINTER(_OgMesh), C.c_double,
                                          C.c_int, C.POINTER(Counters)]
            lib.oracle_voxels.restype = C.c_int
            lib.oracle_voxels_ex.argtypes = [C.POINTER(_OgGrid), C.POINTER(_OgMesh), C.c_double, C.c_int, C.c_int,
                                             C.POINTER(C.c_double), C.POINTER(Counters)]
            lib.oracle_voxels_ex.restype = C.c_int
            lib.oracle_annihilation.argtypes = [C.POINTER(_OgGrid), C.POINTER(_OgMesh), C.c_double, C.c_int,
                                                C.POINTER(Counters)]
            lib.oracle_annihilation.restype = C.c_int
        else:
            lib.psi_voxels.argtypes = [C.POINTER(_PsiGrid), C.POINTER(_PsiMesh), C.c_void_p,
                                       C.c_int, C.c_double, C.c_int]
            lib.psi_voxels.restype = None
        _libs[kind] = lib
    return _libs[kind]


def available(kind: str) -> bool:
    return os.path.exists(_PATHS[kind])


@contextlib.contextmanager
def _quiet_stdout():
    """The reference prints a progress line per 1024 elements (src/cpsi.c:82-83)."""
    import sys
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    try:
        os.dup2(devnull, 1)
        yield
    finally:
        libc = C.CDLL(None)
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def new_fields(n, fields):
    n = tuple(int(v) for v in n)
    shapes = {"m": n, "x": n + (3,), "v": n + (3,), "xx": n + (3, 3), "xv": n + (3, 3), "vv": n + (3, 3)}
    out = {"m": np.zeros(shapes["m"])}
    for f in fields:
        f = "xv" if f == "vx" else f
        out[f] = np.zeros(shapes[f])
    return out


def voxelize(kind, n, bounds, pos, conn, vel=None, mass=None, periodic_box=None, fields=(),
             reftol=1.0, maxlvl=0, out=None, counters=False, refine_mode=0, refine_cell=None, mode="density"):
    """Run the density (or, mode='annihilation', the annihilation) path of the
    chosen back end.

    pos (npart,3) f64, conn (nelem, 4|8) i32, vel like pos (zeros if None),
    mass (nelem,) (ones if None).  ``out`` (a dict of field arrays) is
    accumulated into, as the reference accumulates into grid.fields.
    """
    if refine_mode and kind == "reference":
        raise ValueError("the reference has only the midpoint refinement criterion")
    lib = _lib(kind)
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    conn = conn.reshape(conn.shape[0], -1)
    npart, nelem, et = pos.shape[0], conn.shape[0], conn.shape[1]
    vel = np.zeros_like(pos) if vel is None else np.ascontiguousarray(vel, dtype=np.float64).reshape(-1, 3)
    mass = np.ones(nelem) if mass is None else np.ascontiguousarray(mass, dtype=np.float64).reshape(-1)
    if out is None:
        out = new_fields(n, fields)
    n = [int(v) for v in n]
    lo = [float(v) for v in bounds[0]]
    hi = [float(v) for v in bounds[1]]
    d = [(hi[i] - lo[i]) / n[i] for i in range(3)]  # src/PSI.c:111-113
    box = periodic_box if periodic_box is not None else ((0.0,) * 3, (0.0,) * 3)
    for f, a in out.items():
        assert a.dtype == np.float64 and a.flags.c_contiguous, f
    ptrs = [_dp(out.get(f)) for f in FIELD_NAMES]
    if kind != "reference":
        g = _OgGrid()
        g.n[:] = n
        g.win[0][:] = lo
        g.win[1][:] = hi
        g.d[:] = d
        for i, p in enumerate(ptrs):
            g.f[i] = p
        m = _OgMesh(elemtype=et, npart=npart, nelem=nelem, pos=_dp(pos), vel=_dp(vel), mass=_dp(mass),
                    conn=conn.ctypes.data_as(C.POINTER(C.c_int)), periodic=int(periodic_box is not None))
        m.box[0][:] = [float(v) for v in box[0]]
        m.box[1][:] = [float(v) for v in box[1]]
        cnt = Counters()
        if mode == "annihilation":
            if refine_mode:
                raise ValueError("annihilation takes the midpoint refinement criterion")
            rc = lib.oracle_annihilation(C.byref(g), C.byref(m), float(reftol), int(maxlvl), C.byref(cnt))
        elif refine_mode:
            lag = (C.c_double * 3)(*[float(v) for v in refine_cell])
            rc = lib.oracle_voxels_ex(C.byref(g), C.byref(m), float(reftol), int(maxlvl), int(refine_mode), lag,
                                      C.byref(cnt))
        else:
            rc = lib.oracle_voxels(C.byref(g), C.byref(m), float(reftol), int(maxlvl), C.byref(cnt))
        if rc != 0:
            raise RuntimeError("oracle_voxels failed")
        return (out, cnt.as_dict()) if counters else out
    g = _PsiGrid(type=0, dim=3)
    g.n[:] = n
    g.window[0][:] = lo
    g.window[1][:] = hi
    g.d[:] = d
    for i, p in enumerate(ptrs):
        if p is not None:
            g.fields[i] = p
    m = _PsiMesh(elemtype=et, dim=3, pos=_dp(pos), vel=_dp(vel), mass=_dp(mass), npart=npart, nelem=nelem,
                 connectivity=conn.ctypes.data_as(C.POINTER(C.c_int)), periodic=int(periodic_box is not None))
    m.box[0][:] = [float(v) for v in box[0]]
    m.box[1][:] = [float(v) for v in box[1]]
    with _quiet_stdout():
        lib.psi_voxels(C.byref(g), C.byref(m), None, 1 if mode == "annihilation" else 0, float(reftol), int(maxlvl))
    return (out, None) if counters else out


def block_connectivity(nside, periodic):
    """Trilinear connectivity of a block mesh, as PSI.Mesh(loader='block') builds it
    (src/PSI.c:553-560, :636-656): element (i,j,k) -> vertices 4ii+2jj+kk."""
    nx, ny, nz = (int(v) for v in nside)
    ne = (nx, ny, nz) if periodic else (nx - 1, ny - 1, nz - 1)
    i, j, k = np.meshgrid(np.arange(ne[0]), np.arange(ne[1]), np.arange(ne[2]), indexing="ij")
    conn = np.empty(ne + (8,), dtype=np.int32)
    for ii in range(2):
        for jj in range(2):
            for kk in range(2):
                conn[..., 4 * ii + 2 * jj + kk] = (ny * nz * ((i + ii) % nx) + nz * ((j + jj) % ny)
                                                   + ((k + kk) % nz))
    return conn.reshape(-1, 8)


# ---- snapshot loaders (src/mesh.c:35-302) ----
def _gevolution_tile_tables():
    """The 4^3-tile numbering of src/mesh.c:166-168, rebuilt: slot s of a tile
    holds the particle at 2*G(s // 8) + G(s % 8), G the 3-bit reflected Gray
    code read as (i, j, k) bits, most significant first.  Returns
    (slot -> (i,j,k), [i,j,k] -> slot)."""
    def g3(v):
        gv = v ^ (v >> 1)
        return np.array([(gv >> 2) & 1, (gv >> 1) & 1, gv & 1])

    to_cube = np.array([2 * g3(s // 8) + g3(s % 8) for s in range(64)], dtype=np.int64)
    to_flat = np.full((4, 4, 4), -1, dtype=np.int64)
    for s in range(64):
        to_flat[tuple(to_cube[s])] = s
    assert (to_flat >= 0).all()
    return to_cube, to_flat


def load_snapshot(kind, path, flavour="gadget2"):
    """pos, vel (npart,3), mass (npart,), connectivity (npart,8) int32 and the
    box size of a Gadget-2 format-1 snapshot, as PSI.Mesh(loader=flavour) reads
    it.  kind 'restatement': numpy, following src/mesh.c:64-160 ('gadget2') and
    :163-302 ('gevolution'); kind 'reference': the reference's own
    peek_gadget2 + load_gadget2 / load_gevolution from _ref/libpsiref.so."""
    if kind == "reference":
        lib = _lib("reference")
        m = _PsiMesh()
        with _quiet_stdout():
            ok = lib.peek_gadget2(C.byref(m), path.encode())
        if not ok:
            raise ValueError("peek_gadget2 failed")
        npart = m.npart
        pos, vel = np.zeros((npart, 3)), np.zeros((npart, 3))
        mass, conn = np.zeros(npart), np.zeros((npart, 8), dtype=np.int32)
        m.pos, m.vel, m.mass = _dp(pos), _dp(vel), _dp(mass)
        m.connectivity = conn.ctypes.data_as(C.POINTER(C.c_int))
        fn = lib.load_gadget2 if flavour == "gadget2" else lib.load_gevolution
        with _quiet_stdout():
            ok = fn(C.byref(m), path.encode())
        if not ok:
            raise ValueError(f"{fn.__name__} failed")
        return pos, vel, mass, conn, m.box[1][0]
    raw = open(path, "rb").read()
    hdr = raw[4:260]
    npart = int(np.frombuffer(hdr, np.int32, 6, 0)[1])
    mass1 = float(np.frombuffer(hdr, np.float64, 6, 24)[1])
    box = float(np.frombuffer(hdr, np.float64, 1, 128)[0])
    at = 264 + 4
    tpos = np.frombuffer(raw, np.float32, 3 * npart, at).reshape(npart, 3)
    at += 12 * npart + 8
    tvel = np.frombuffer(raw, np.float32, 3 * npart, at).reshape(npart, 3)
    at += 12 * npart + 8
    idt = np.int32 if flavour == "gadget2" else np.int64
    tid = np.frombuffer(raw, idt, npart, at).astype(np.int64)
    pos, vel = np.zeros((npart, 3)), np.zeros((npart, 3))
    pos[tid] = tpos
    vel[tid] = tvel
    mass = np.full(npart, mass1 / npart)
    nside = int(np.floor((npart + 0.5) ** (1.0 / 3.0)))
    if flavour == "gadget2":
        conn = block_connectivity((nside,) * 3, True)
    else:
        to_cube, to_flat = _gevolution_tile_tables()
        tn = nside // 4
        p = np.arange(npart)
        t = p // 64
        tile = np.stack([t % tn, (t // tn) % tn, t // (tn * tn)], axis=1)
        cube = to_cube[p % 64]
        conn = np.empty((npart, 8), dtype=np.int32)
        for ii in range(2):
            for jj in range(2):
                for kk in range(2):
                    q = cube + np.array([ii, jj, kk])
                    dt, q = q // 4, q % 4
                    tt = (tile + dt) % tn
                    flat = tt[:, 0] + tn * tt[:, 1] + tn * tn * tt[:, 2]
                    conn[:, 4 * ii + 2 * jj + kk] = 64 * flat + to_flat[q[:, 0], q[:, 1], q[:, 2]]
    return pos, vel, mass, conn, box


# ---- element queries and phase-space samples (src/rtree.c, src/cpsi.c:177-275) ----
class _PsiRtree(C.Structure):
    _fields_ = [("root", C.c_int), ("depth", C.c_int), ("allnodes", C.c_void_p), ("nodecap", C.c_int),
                ("nnodes", C.c_int)]


class _Rvec(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


def _meshes(pos, conn, vel=None, mass=None, periodic_box=None):
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    conn = conn.reshape(conn.shape[0], -1)
    vel = np.zeros_like(pos) if vel is None else np.ascontiguousarray(vel, dtype=np.float64).reshape(-1, 3)
    mass = np.ones(conn.shape[0]) if mass is None else np.ascontiguousarray(mass, dtype=np.float64).reshape(-1)
    box = periodic_box if periodic_box is not None else ((0.0,) * 3, (0.0,) * 3)
    keep = (pos, conn, vel, mass)
    og = _OgMesh(elemtype=conn.shape[1], npart=pos.shape[0], nelem=conn.shape[0], pos=_dp(pos), vel=_dp(vel),
                 mass=_dp(mass), conn=conn.ctypes.data_as(C.POINTER(C.c_int)), periodic=int(periodic_box is not None))
    ps = _PsiMesh(elemtype=conn.shape[1], dim=3, pos=_dp(pos), vel=_dp(vel), mass=_dp(mass), npart=pos.shape[0],
                  nelem=conn.shape[0], connectivity=conn.ctypes.data_as(C.POINTER(C.c_int)),
                  periodic=int(periodic_box is not None))
    for m in (og, ps):
        m.box[0][:] = [float(v) for v in box[0]]
        m.box[1][:] = [float(v) for v in box[1]]
    return og, ps, keep, box


def tree_window(periodic_box):
    """The cull window of PSI.RStarTree(mesh) (src/PSI.c:865-896)."""
    if periodic_box is not None:
        return tuple(tuple(float(v) for v in b) for b in periodic_box)
    return ((-1.0e30,) * 3, (1.0e30,) * 3)


def query_elements(kind, pos, conn, window, box, periodic_box=None):
    """Element indices whose unwrapped box touches `box`, over the elements that
    survive the cull against `window`: PSI.RStarTree(...).query (src/PSI.c:817-862)."""
    og, ps, keep, _ = _meshes(pos, conn, periodic_box=periodic_box)
    lib = _lib(kind)
    win = np.ascontiguousarray(window, dtype=np.float64).reshape(2, 3)
    q = np.ascontiguousarray(box, dtype=np.float64).reshape(2, 3)
    if kind != "reference":
        lib.oracle_query.restype = C.c_longlong
        n = lib.oracle_query(C.byref(og), _dp(win), _dp(q), None, C.c_longlong(0))
        out = np.zeros(max(n, 1), dtype=np.int32)
        lib.oracle_query(C.byref(og), _dp(win), _dp(q), out.ctypes.data_as(C.POINTER(C.c_int)), C.c_longlong(n))
        return out[:n]
    tree = _PsiRtree()
    qry = C.create_string_buffer(1 << 15)
    res = []
    with _quiet_stdout():
        lib.psi_rtree_from_mesh(C.byref(tree), C.byref(ps), _dp(win))
        lib.psi_rtree_query_init(qry, C.byref(tree), _dp(q))
        e = C.c_int()
        while lib.psi_rtree_query_next(qry, C.byref(e)):
            res.append(e.value)
        lib.psi_rtree_destroy(C.byref(tree))
    return np.array(res, dtype=np.int32)


def sample_vdf(kind, pos, conn, point, vel=None, mass=None, periodic_box=None, window=None, reftol=1.0, maxlvl=0):
    """PSI.VDF(mesh, sample_pos, tree, ...) (src/PSI.c:1022-1057): densities (n,) and
    velocities (n, 3) of the streams at `point`.  window None: the tree PSI.VDF
    builds itself, over the cull window mesh.box (zero for an open mesh); else the
    window of the given tree (tree_window)."""
    og, ps, keep, box = _meshes(pos, conn, vel, mass, periodic_box)
    lib = _lib(kind)
    s = np.ascontiguousarray(point, dtype=np.float64).reshape(3)
    win = np.ascontiguousarray(box if window is None else window, dtype=np.float64).reshape(2, 3)
    if kind != "reference":
        f = lib.oracle_sample_vdf
        f.restype = C.c_longlong
        f.argtypes = [C.POINTER(_OgMesh), C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double, C.c_int,
                      C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_longlong]
        n = f(C.byref(og), _dp(win), _dp(s), float(reftol), int(maxlvl), None, None, 0)
        if n < 0:
            raise ValueError("oracle_sample_vdf: unsupported element type")
        rho, v = np.zeros(max(n, 1)), np.zeros((max(n, 1), 3))
        f(C.byref(og), _dp(win), _dp(s), float(reftol), int(maxlvl), _dp(rho), _dp(v), n)
        return rho[:n], v[:n]
    tree = _PsiRtree() if window is not None else None
    rp, vp, ns = C.POINTER(C.c_double)(), C.POINTER(C.c_double)(), C.c_int()
    libc = C.CDLL(None)
    with _quiet_stdout():
        if tree is not None:
            lib.psi_rtree_from_mesh(C.byref(tree), C.byref(ps), _dp(win))
        lib.psi_sample_vdf.argtypes = [_Rvec, C.POINTER(_PsiMesh), C.c_void_p, C.POINTER(C.POINTER(C.c_double)),
                                       C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_int), C.c_double, C.c_int]
        lib.psi_sample_vdf(_Rvec(*s), C.byref(ps), C.cast(C.byref(tree), C.c_void_p) if tree is not None else None,
                           C.byref(rp), C.byref(vp), C.byref(ns), float(reftol), int(maxlvl))
        if tree is not None:
            lib.psi_rtree_destroy(C.byref(tree))
    n = ns.value
    rho = np.ctypeslib.as_array(rp, shape=(n,)).copy() if n else np.zeros(0)
    v = np.ctypeslib.as_array(vp, shape=(n, 3)).copy() if n else np.zeros((0, 3))
    libc.free(C.cast(rp, C.c_void_p))
    libc.free(C.cast(vp, C.c_void_p))
    return rho, v


def sample_vdf_many(kind, pos, conn, points, vel=None, mass=None, periodic_box=None, window=None, reftol=1.0,
                    maxlvl=0):
    """sample_vdf at many points: for the reference, one tree built once (the
    tree a PSI.RStarTree holds) and psi_sample_vdf per point.  Returns the list
    of (rho, vel) per point and the seconds spent sampling (tree build excluded)."""
    import time

    if kind != "reference":
        t0 = time.perf_counter()
        res = [sample_vdf(kind, pos, conn, p, vel, mass, periodic_box, window, reftol, maxlvl) for p in points]
        return res, time.perf_counter() - t0
    og, ps, keep, box = _meshes(pos, conn, vel, mass, periodic_box)
    lib = _lib(kind)
    win = np.ascontiguousarray(box if window is None else window, dtype=np.float64).reshape(2, 3)
    tree = _PsiRtree()
    libc = C.CDLL(None)
    lib.psi_sample_vdf.argtypes = [_Rvec, C.POINTER(_PsiMesh), C.c_void_p, C.POINTER(C.POINTER(C.c_double)),
                                   C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_int), C.c_double, C.c_int]
    res = []
    with _quiet_stdout():
        lib.psi_rtree_from_mesh(C.byref(tree), C.byref(ps), _dp(win))
        t0 = time.perf_counter()
        for p in np.asarray(points, dtype=np.float64).reshape(-1, 3):
            rp, vp, ns = C.POINTER(C.c_double)(), C.POINTER(C.c_double)(), C.c_int()
            lib.psi_sample_vdf(_Rvec(*p), C.byref(ps), C.cast(C.byref(tree), C.c_void_p), C.byref(rp), C.byref(vp),
                               C.byref(ns), float(reftol), int(maxlvl))
            n = ns.value
            res.append((np.ctypeslib.as_array(rp, shape=(n,)).copy() if n else np.zeros(0),
                        np.ctypeslib.as_array(vp, shape=(n, 3)).copy() if n else np.zeros((0, 3))))
            libc.free(C.cast(rp, C.c_void_p))
            libc.free(C.cast(vp, C.c_void_p))
        secs = time.perf_counter() - t0
        lib.psi_rtree_destroy(C.byref(tree))
    return res, secs
