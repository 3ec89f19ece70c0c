"""ctypes binding of include/psi_b200.h for callers that hold device memory.

``voxels_device`` runs psib_voxels in PSIB_DEVICE mode on buffers that already
live on the GPU (torch CUDA tensors here, raw device pointers in general) and on
the caller's CUDA stream.  It is also the template of the binding a maintainer
of the reference would add to call the library from Python without the PSI
extension: one ctypes structure per C struct of the header, one argtypes line
per entry point, and a status code turned into an exception.
"""
from __future__ import annotations

import ctypes as C

from . import lib

PSIB_FP64, PSIB_MIXED, PSIB_FP64_CENTRAL = 0, 1, 2
PRECISIONS = {"fp64": PSIB_FP64, "mixed": PSIB_MIXED, "fp64-central": PSIB_FP64_CENTRAL}
PSIB_HOST, PSIB_DEVICE = 0, 1
FIELDS = ("m", "x", "v", "xx", "xv", "vv")
COMPONENTS = {"m": 1, "x": 3, "v": 3, "xx": 9, "xv": 9, "vv": 9}


class Grid(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("window", (C.c_double * 3) * 2), ("d", C.c_double * 3),
                ("fields", C.c_void_p * 6)]


class Mesh(C.Structure):
    _fields_ = [("elemtype", C.c_int), ("npart", C.c_longlong), ("nelem", C.c_longlong), ("pos", C.c_void_p),
                ("vel", C.c_void_p), ("mass", C.c_void_p), ("connectivity", C.c_void_p),
                ("block_dims", C.c_int * 3), ("periodic", C.c_int), ("box", (C.c_double * 3) * 2)]


class Stats(C.Structure):
    _fields_ = [("elements_kept", C.c_longlong), ("tets", C.c_longlong), ("tet_images", C.c_longlong),
                ("fragments", C.c_longlong), ("frag_verts", C.c_longlong), ("splits", C.c_longlong),
                ("passes", C.c_int), ("chunks", C.c_int), ("ms_total", C.c_float), ("ms_clip", C.c_float),
                ("ms_tess", C.c_float), ("ms_final", C.c_float), ("clip_launches", C.c_longlong),
                ("kernel_launches", C.c_longlong), ("walk_bytes", C.c_longlong),
                ("corrected_items", C.c_longlong), ("accumulation", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("deterministic", C.c_int), ("memory", C.c_int), ("device", C.c_int),
                ("stream", C.c_void_p), ("stats", C.POINTER(Stats)), ("refine_mode", C.c_int),
                ("refine_cell", C.c_double * 3), ("queue_voxels", C.c_longlong), ("capture", C.c_int),
                ("order_cell_bits", C.c_int)]


lib.psib_voxels.argtypes = [C.POINTER(Grid), C.POINTER(Mesh), C.c_int, C.c_double, C.c_int, C.POINTER(Options)]
lib.psib_voxels.restype = C.c_int
lib.psib_voxels_adjoint.argtypes = [C.POINTER(Grid), C.POINTER(Mesh), C.c_double, C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.POINTER(Options)]
lib.psib_voxels_adjoint.restype = C.c_int
lib.psib_voxels_batch.argtypes = [C.POINTER(Grid), C.POINTER(Mesh), C.c_int, C.c_int, C.c_double, C.c_int,
                                  C.POINTER(Options)]
lib.psib_voxels_batch.restype = C.c_int
lib.psib_query_elements.argtypes = [C.POINTER(Mesh), C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p,
                                    C.c_longlong, C.POINTER(Options)]
lib.psib_query_elements.restype = C.c_int
lib.psib_sample_vdf.argtypes = [C.POINTER(Mesh), C.c_void_p, C.c_void_p, C.c_longlong, C.c_double, C.c_int, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_longlong, C.POINTER(Options)]
lib.psib_sample_vdf.restype = C.c_int
lib.psib_voxels_adjoint_fields.argtypes = [C.POINTER(Grid), C.POINTER(Grid), C.POINTER(Mesh), C.c_double, C.c_int,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Options)]
lib.psib_voxels_adjoint_fields.restype = C.c_int
lib.psib_measure_fma_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
lib.psib_measure_fma_peak.restype = C.c_int
lib.psib_capture_status.restype = C.c_int
lib.psib_last_error.restype = C.c_char_p
lib.psib_release_device_memory.restype = C.c_int


class PsibError(RuntimeError):
    def __init__(self, code: int):
        self.code = code
        super().__init__(f"psib_voxels failed (code {code}): {lib.psib_last_error().decode()}")


def measure_fma_peak(precision="fp64") -> float:
    """This GPU's FMA issue rate in TFLOP/s, 'fp64' or 'fp32' (psib_measure_fma_peak)."""
    out = C.c_double(0.0)
    rc = lib.psib_measure_fma_peak(PSIB_FP64 if precision == "fp64" else PSIB_MIXED, C.byref(out))
    if rc != 0:
        raise PsibError(rc)
    return out.value


def make_grid(n, bounds, field_ptrs: dict) -> Grid:
    g = Grid()
    g.n[:] = [int(v) for v in n]
    for i in range(3):
        g.window[0][i] = float(bounds[0][i])
        g.window[1][i] = float(bounds[1][i])
        g.d[i] = (g.window[1][i] - g.window[0][i]) / g.n[i]  # as src/PSI.c:111-113
    for i, f in enumerate(FIELDS):
        g.fields[i] = field_ptrs.get(f)
    return g


def make_mesh(npart, nelem, pos_ptr, vel_ptr=None, mass_ptr=None, conn_ptr=None, elemtype=8, block_dims=None,
              periodic_box=None) -> Mesh:
    m = Mesh(elemtype=elemtype, npart=int(npart), nelem=int(nelem), pos=pos_ptr, vel=vel_ptr, mass=mass_ptr,
             connectivity=conn_ptr)
    if block_dims is not None:
        m.block_dims[:] = [int(v) for v in block_dims]
    if periodic_box is not None:
        m.periodic = 1
        for i in range(3):
            m.box[0][i] = float(periodic_box[0][i])
            m.box[1][i] = float(periodic_box[1][i])
    return m


REFINE = {"midpoint": 0, "stretch": 1}
MODES = {"density": 0, "annihilation": 1}


def voxels(grid: Grid, mesh: Mesh, precision=PSIB_FP64, deterministic=False, memory=PSIB_DEVICE, stream=None,
           refine_tolerance=1.0, refine_max_lvl=0, refine_criterion="midpoint", refine_cell=None,
           mode="density", order_cell_bits=0) -> dict:
    st = Stats()
    o = Options(precision=precision, deterministic=int(bool(deterministic)), memory=memory, device=-1,
                stream=stream, stats=C.pointer(st), refine_mode=REFINE[refine_criterion],
                order_cell_bits=int(order_cell_bits))
    if refine_cell is not None:
        o.refine_cell[:] = [float(v) for v in refine_cell]
    rc = lib.psib_voxels(C.byref(grid), C.byref(mesh), MODES[mode], float(refine_tolerance), int(refine_max_lvl),
                         C.byref(o))
    if rc != 0:
        raise PsibError(rc)
    return st.as_dict()


def voxels_device(fields: dict, n, bounds, pos, vel=None, mass=None, connectivity=None, block_dims=None,
                  periodic_box=None, precision="fp64", deterministic=False, refine_tolerance=1.0, refine_max_lvl=0,
                  stream=None, refine_criterion="midpoint", refine_cell=None, mode="density",
                  order_cell_bits=0) -> dict:
    """Deposit on device-resident torch tensors (mode 'density', or
    'annihilation': m gains the integral of rho_0 rho_1 over overlapping tets).

    fields: {"m": (nx,ny,nz) float64 CUDA tensor, "x": (...,3), ...}; pos/vel:
    (npart,3) float64; mass: (nelem,) float64; connectivity: (nelem, 4|8) int32
    or None with block_dims for a block lattice.  Runs on `stream` (a
    torch.cuda.Stream; default: the current stream)."""
    import torch

    for f, t in fields.items():
        assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous(), f
    ptr = {f: t.data_ptr() for f, t in fields.items()}
    g = make_grid(n, bounds, ptr)
    m = mesh_from_tensors(pos, vel, mass, connectivity, block_dims, periodic_box)
    s = stream if stream is not None else torch.cuda.current_stream()
    return voxels(g, m, PRECISIONS[precision], deterministic, PSIB_DEVICE,
                  C.c_void_p(s.cuda_stream), refine_tolerance, refine_max_lvl, refine_criterion, refine_cell, mode,
                  order_cell_bits)


def mesh_from_tensors(pos, vel=None, mass=None, connectivity=None, block_dims=None, periodic_box=None) -> Mesh:
    """A psib_mesh over contiguous tensors (or arrays with data_ptr())."""
    npart = pos.numel() // 3
    if connectivity is not None:
        elemtype, nelem = connectivity.shape[-1], connectivity.numel() // connectivity.shape[-1]
    else:
        elemtype = 8
        nelem = 1
        for b in block_dims:
            nelem *= b if periodic_box is not None else b - 1
    return make_mesh(npart, nelem, pos.data_ptr(), vel.data_ptr() if vel is not None else None,
                     mass.data_ptr() if mass is not None else None,
                     connectivity.data_ptr() if connectivity is not None else None, elemtype, block_dims, periodic_box)


def adjoint_device(grad_m, n, bounds, pos, grad_pos, mass=None, connectivity=None, block_dims=None,
                   periodic_box=None, grad_mass=None, stream=None, refine_tolerance=1.0, refine_max_lvl=0) -> dict:
    """Backward pass of the m field on device-resident torch tensors.

    grad_m: (nx,ny,nz) float64 CUDA tensor, dL/dm.  Adds dL/dpos to grad_pos
    ((npart,3) float64) and, if given, dL/dmass to grad_mass ((nelem,)).  The
    refinement arguments are those of the forward deposit (midpoint criterion)."""
    import torch

    for t in (grad_m, pos, grad_pos) + ((grad_mass,) if grad_mass is not None else ()):
        assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
    g = make_grid(n, bounds, {"m": grad_m.data_ptr()})
    m = mesh_from_tensors(pos, None, mass, connectivity, block_dims, periodic_box)
    s = stream if stream is not None else torch.cuda.current_stream()
    st = Stats()
    o = Options(precision=PSIB_FP64, deterministic=0, memory=PSIB_DEVICE, device=-1,
                stream=C.c_void_p(s.cuda_stream), stats=C.pointer(st))
    rc = lib.psib_voxels_adjoint(C.byref(g), C.byref(m), float(refine_tolerance), int(refine_max_lvl),
                                 grad_pos.data_ptr(), None,
                                 grad_mass.data_ptr() if grad_mass is not None else None, C.byref(o))
    if rc != 0:
        raise PsibError(rc)
    return st.as_dict()


def adjoint_fields_device(grads: dict, fwd: dict, n, bounds, pos, grad_pos, vel=None, mass=None, connectivity=None,
                          block_dims=None, periodic_box=None, grad_vel=None, grad_mass=None, stream=None,
                          refine_tolerance=1.0, refine_max_lvl=0) -> dict:
    """Backward pass of every field (psib_voxels_adjoint_fields) on device tensors.

    fwd: the fields of the forward deposit into zeroed fields ({"m": ..., "x": ...});
    grads: dL/d(field) for any of them (missing: 0).  Adds dL/dpos to grad_pos and,
    if given, dL/dvel to grad_vel ((npart,3)) and dL/dmass to grad_mass ((nelem,)).
    The refinement arguments are those of the forward deposit (midpoint criterion)."""
    import torch

    for t in list(grads.values()) + list(fwd.values()) + [pos, grad_pos] + \
            [t for t in (vel, grad_vel, grad_mass) if t is not None]:
        assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
    g = make_grid(n, bounds, {f: t.data_ptr() for f, t in grads.items()})
    f = make_grid(n, bounds, {k: t.data_ptr() for k, t in fwd.items()})
    m = mesh_from_tensors(pos, vel, mass, connectivity, block_dims, periodic_box)
    s = stream if stream is not None else torch.cuda.current_stream()
    st = Stats()
    o = Options(precision=PSIB_FP64, deterministic=0, memory=PSIB_DEVICE, device=-1,
                stream=C.c_void_p(s.cuda_stream), stats=C.pointer(st))
    rc = lib.psib_voxels_adjoint_fields(C.byref(g), C.byref(f), C.byref(m), float(refine_tolerance),
                                        int(refine_max_lvl), grad_pos.data_ptr(),
                                        grad_vel.data_ptr() if grad_vel is not None else None,
                                        grad_mass.data_ptr() if grad_mass is not None else None, C.byref(o))
    if rc != 0:
        raise PsibError(rc)
    return st.as_dict()


def voxels_batch_device(cutouts: list, precision="fp64", refine_tolerance=1.0, refine_max_lvl=0,
                        refine_criterion="midpoint", refine_cell=None, stream=None, queue_voxels=0,
                        deterministic=False, capture=0, order_cell_bits=0) -> dict:
    """Many independent deposits in one pass (psib_voxels_batch).

    cutouts: dicts with the arguments of voxels_device -- fields, n, bounds,
    pos and optionally vel, mass, connectivity, block_dims, periodic_box --
    all on the GPU; every cutout must ask for the same fields."""
    import torch

    nb = len(cutouts)
    grids = (Grid * nb)()
    meshes = (Mesh * nb)()
    for b, c in enumerate(cutouts):
        for f, t in c["fields"].items():
            assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous(), f
        grids[b] = make_grid(c["n"], c["bounds"], {f: t.data_ptr() for f, t in c["fields"].items()})
        meshes[b] = mesh_from_tensors(c["pos"], c.get("vel"), c.get("mass"), c.get("connectivity"),
                                      c.get("block_dims"), c.get("periodic_box"))
    s = stream if stream is not None else torch.cuda.current_stream()
    st = Stats()
    o = Options(precision=PRECISIONS[precision], deterministic=int(bool(deterministic)), memory=PSIB_DEVICE,
                device=-1, stream=C.c_void_p(s.cuda_stream), stats=C.pointer(st),
                refine_mode=REFINE[refine_criterion], queue_voxels=int(queue_voxels), capture=int(capture),
                order_cell_bits=int(order_cell_bits))
    if refine_cell is not None:
        o.refine_cell[:] = [float(v) for v in refine_cell]
    rc = lib.psib_voxels_batch(grids, meshes, nb, 0, float(refine_tolerance), int(refine_max_lvl), C.byref(o))
    if rc != 0:
        raise PsibError(rc)
    return st.as_dict()


def capture_status() -> int:
    """psib_capture_status: the status that capture-mode calls left on the current device (0: ok)."""
    return lib.psib_capture_status()


def capture_batch(cutouts: list, precision="mixed", queue_voxels=0, **kw):
    """A batch call recorded in a torch CUDA graph: one plan call (options.capture = 1,
    which also deposits once), then one capture-mode call (capture = 2) recorded
    and returned as a torch.cuda.CUDAGraph.  graph.replay() repeats the deposit on
    the cutouts' current particle arrays and fields (it adds to the fields, as a
    call does); check capture_status() after replays."""
    import torch

    voxels_batch_device(cutouts, precision=precision, queue_voxels=queue_voxels, capture=1, **kw)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        voxels_batch_device(cutouts, precision=precision, queue_voxels=queue_voxels, capture=2,
                            stream=torch.cuda.current_stream(), **kw)
    return g


def autotune_batch(cutouts: list, candidates=(8 << 20, 16 << 20, 32 << 20, 64 << 20), precision="mixed",
                   repeats=2, tiles=(7, 5, 3, -1), **kw) -> dict:
    """Pick the launch parameters of a batch that will be deposited many times (the
    same cutouts with new positions, say): the queue capacity
    (psib_options.queue_voxels) and the spatial tile of the work order
    (psib_options.order_cell_bits: 2^b coarse cells over each grid).

    Each pair is timed with CUDA events over `repeats` batch calls after one
    warm-up call; the fields of the cutouts are zeroed afterwards.  Returns
    {"queue_voxels": ..., "order_cell_bits": ..., "ms": ...}, whose first two
    entries go to voxels_batch_device."""
    import torch

    best = {"queue_voxels": 0, "order_cell_bits": 0, "ms": float("inf")}
    stream = torch.cuda.current_stream()
    for cap in candidates:
        for bits in tiles:
            try:
                voxels_batch_device(cutouts, precision=precision, queue_voxels=cap, order_cell_bits=bits, **kw)
            except PsibError:
                continue  # e.g. not enough memory for this capacity
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(repeats):
                voxels_batch_device(cutouts, precision=precision, queue_voxels=cap, order_cell_bits=bits, **kw)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / repeats
            if ms < best["ms"]:
                best = {"queue_voxels": cap, "order_cell_bits": bits, "ms": ms}
    for c in cutouts:
        for t in c["fields"].values():
            t.zero_()
    return best


def tree_window(periodic_box=None):
    """The cull window of PSI.RStarTree(mesh): the periodic box, or +-1e30."""
    if periodic_box is not None:
        return (tuple(float(v) for v in periodic_box[0]), tuple(float(v) for v in periodic_box[1]))
    return ((-1.0e30,) * 3, (1.0e30,) * 3)


def _window_array(window):
    import numpy as np

    return np.ascontiguousarray(np.array([list(window[0]), list(window[1])], dtype=np.float64))


def sample_vdf(points, pos, connectivity=None, vel=None, mass=None, block_dims=None, periodic_box=None, window=None,
               refine_tolerance=1.0, refine_max_lvl=0):
    """Phase-space samples at many points at once (psib_sample_vdf): the
    batched PSI.VDF.  numpy arrays (host memory) or CUDA tensors (device
    memory, on the current stream).  window: a tree's cull window (default:
    tree_window(periodic_box), as PSI.RStarTree(mesh) has).  Returns
    (offsets (npoints + 1,), rho (n,), vel (n, 3)); point p's samples are
    [offsets[p], offsets[p + 1])."""
    import numpy as np

    device = hasattr(points, "is_cuda") and points.is_cuda
    win = _window_array(tree_window(periodic_box) if window is None else window)
    if device:
        m = mesh_from_tensors(pos, vel, mass, connectivity, block_dims, periodic_box)
    else:
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        mass = None if mass is None else np.ascontiguousarray(mass, dtype=np.float64)
        connectivity = None if connectivity is None else np.ascontiguousarray(connectivity, dtype=np.int32)
        npart = pos.size // 3
        if connectivity is not None:
            et, nelem = connectivity.shape[-1], connectivity.size // connectivity.shape[-1]
        else:
            et, nelem = 8, int(np.prod([b if periodic_box is not None else b - 1 for b in block_dims]))
        m = make_mesh(npart, nelem, pos.ctypes.data, None if vel is None else vel.ctypes.data,
                      None if mass is None else mass.ctypes.data,
                      None if connectivity is None else connectivity.ctypes.data, et, block_dims, periodic_box)
    npts = points.shape[0]
    if device:
        import torch

        s = torch.cuda.current_stream()
        o = Options(precision=PSIB_FP64, memory=PSIB_DEVICE, device=-1, stream=C.c_void_p(s.cuda_stream))
        off = torch.zeros(npts + 1, dtype=torch.int64, device=points.device)
        rc = lib.psib_sample_vdf(C.byref(m), win.ctypes.data, points.data_ptr(), npts, float(refine_tolerance),
                                 int(refine_max_lvl), off.data_ptr(), None, None, 0, C.byref(o))
        if rc != 0:
            raise PsibError(rc)
        n = int(off[-1].item())
        rho = torch.empty(max(n, 1), dtype=torch.float64, device=points.device)
        v = torch.empty((max(n, 1), 3), dtype=torch.float64, device=points.device)
        if n:
            rc = lib.psib_sample_vdf(C.byref(m), win.ctypes.data, points.data_ptr(), npts, float(refine_tolerance),
                                     int(refine_max_lvl), off.data_ptr(), rho.data_ptr(), v.data_ptr(), n, C.byref(o))
            if rc != 0:
                raise PsibError(rc)
        return off, rho[:n], v[:n]
    points = np.ascontiguousarray(points, dtype=np.float64)
    o = Options(precision=PSIB_FP64, memory=PSIB_HOST, device=-1)
    off = np.zeros(npts + 1, dtype=np.int64)
    rc = lib.psib_sample_vdf(C.byref(m), win.ctypes.data, points.ctypes.data, npts, float(refine_tolerance),
                             int(refine_max_lvl), off.ctypes.data, None, None, 0, C.byref(o))
    if rc != 0:
        raise PsibError(rc)
    n = int(off[-1])
    rho, v = np.zeros(max(n, 1)), np.zeros((max(n, 1), 3))
    if n:
        rc = lib.psib_sample_vdf(C.byref(m), win.ctypes.data, points.ctypes.data, npts, float(refine_tolerance),
                                 int(refine_max_lvl), off.ctypes.data, rho.ctypes.data, v.ctypes.data, n, C.byref(o))
        if rc != 0:
            raise PsibError(rc)
    return off, rho[:n], v[:n]
