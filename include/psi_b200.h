/*
 * psi_b200.h -- C ABI of the B200 phase-space-sheet voxelizer (libpsi_b200.so).
 *
 * Plain C types only: pointers, sizes and status codes.  No CUDA, C++ or
 * PyTorch type appears in a signature; the stream is passed as void*.
 *
 * The library replaces the density path of PyPSI:
 *   void psi_voxels(psi_grid* grid, psi_mesh* mesh, psi_rtree* rtree,
 *                   psi_int mode, psi_real reftol, psi_int max_ref_lvl);
 * declared at src/PSI.c:39, defined at src/cpsi.c:41, and called only from
 * PSI_voxels at src/PSI.c:1015.  psib_grid and psib_mesh carry the same data
 * as psi_grid (include/grid.h:46-53) and psi_mesh (include/mesh.h:42-52),
 * with the same array layouts (src/PSI.c:124-186, :399-656).
 *
 * Every entry point returns PSIB_OK (0) or a PSIB_ERR_* code; none exits or
 * aborts.  psib_last_error() gives a message for the last failure on the
 * calling thread.
 */
#ifndef PSI_B200_H
#define PSI_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define PSIB_ABI_VERSION 2

/* status codes */
#define PSIB_OK 0
#define PSIB_ERR_ARG 1         /* invalid argument (shape, type, value) */
#define PSIB_ERR_CUDA 2        /* a CUDA runtime call failed */
#define PSIB_ERR_NOMEM 3       /* device or pinned host allocation failed */
#define PSIB_ERR_OVERFLOW 4    /* a polyhedron outgrew its vertex buffer */
#define PSIB_ERR_INDEX 5       /* connectivity or voxel index out of range */
#define PSIB_ERR_UNSUPPORTED 6 /* a mode the library does not implement */
#define PSIB_ERR_NODEVICE 7    /* no CUDA device is visible */

/* grid field tags, as include/grid.h:37-42 */
#define PSIB_M 0
#define PSIB_X 1
#define PSIB_V 2
#define PSIB_XX 3
#define PSIB_XV 4
#define PSIB_VV 5

/* deposit mode, as include/psi.h:69-70 */
#define PSIB_MODE_DENSITY 0
#define PSIB_MODE_ANNIHILATION 1 /* src/cpsi.c:115-158: adds to m the integral of rho_0 rho_1 over every
                                    pair of overlapping tets (FP64; precision is ignored) */

/* arithmetic of the clip kernel */
#define PSIB_FP64 0  /* the reference's double-precision operation order, no FMA */
#define PSIB_MIXED 1 /* FP32 bisection walk; fragment vertices recomputed in FP64 from their planes,
                        FP64 moments and sums */
#define PSIB_FP64_CENTRAL 2 /* FP64 walk with moments taken about each fragment: more accurate than the
                               reference for tiny fragments, not bit-identical to it */

/* refinement criterion of trilinear elements (psib_options.refine_mode) */
#define PSIB_REFINE_MIDPOINT 0 /* the reference's: an edge midpoint of the trilinear map deviates from the
                                  straight edge by more than refine_tolerance x the smallest cell
                                  (src/refine.c:223-289, src/cpsi.c:63-66) */
#define PSIB_REFINE_STRETCH 1  /* not in the reference: a (sub)cube of level l is refined when an edge along
                                  axis a exceeds refine_tolerance x refine_cell[a] / 2^l, or its volume exceeds
                                  refine_tolerance x the cell volume / 8^l */

/* where the pointers of psib_grid / psib_mesh live */
#define PSIB_HOST 0   /* host memory; the library copies in and out */
#define PSIB_DEVICE 1 /* device memory of the current CUDA device */

/* Cartesian grid.  fields[t] points to nx*ny*nz*{1,3,9} doubles in C order
 * (m: (nx,ny,nz); x,v: (...,3); xx,xv,vv: (...,3,3)) or is NULL when the field
 * is not requested.  fields[PSIB_M] is required.  As in the reference the call
 * ACCUMULATES into the fields: m is a mass sum, x and v mass-weighted means,
 * xx, xv, vv mass-weighted (co)variances (src/geometry.c:164-186). */
typedef struct {
    int n[3];
    double window[2][3];
    double d[3]; /* (window[1]-window[0])/n, as src/PSI.c:111-113 computes it */
    double *fields[6];
} psib_grid;

/* Lagrangian mesh.  pos and vel are npart x 3 doubles (vel may be NULL:
 * zeros), mass is one double per element (NULL: ones).  connectivity is
 * nelem x elemtype ints (elemtype 4: tets, 8: trilinear cubes, 27: triquadratic
 * cubes, as src/PSI.c:439-443 accepts).  With connectivity == NULL and
 * block_dims set, the trilinear block connectivity of src/PSI.c:636-656 is
 * implied (periodic wrap when periodic != 0), and is never materialised. */
typedef struct {
    int elemtype;
    long long npart;
    long long nelem;
    const double *pos;
    const double *vel;
    const double *mass;
    const int *connectivity;
    int block_dims[3];
    int periodic;
    double box[2][3];
} psib_mesh;

/* Work counters and timings of one call (all optional outputs). */
typedef struct {
    long long elements_kept; /* elements surviving the window cull */
    long long tets;          /* tets after refinement, without periodic images */
    long long tet_images;    /* tets including periodic images (work items) */
    long long fragments;     /* (tet image, voxel) pieces with m0 > 0 */
    long long frag_verts;    /* sum of fragment vertex counts */
    long long splits;        /* axis-aligned splits of the bisection */
    int passes;              /* clip passes over the tets (1) */
    int chunks;              /* element chunks the tets were streamed in */
    float ms_total;          /* device time of the whole call, host copies included */
    float ms_clip;           /* device time of the clip kernels */
    float ms_tess;           /* device time of tessellation and ordering */
    float ms_final;          /* device time of the record sort and the field update */
    long long clip_launches; /* launches of the clip kernels */
    long long kernel_launches; /* launches of this library's own kernels (library scans/sorts excluded) */
    long long walk_bytes;    /* bytes the breadth-first walk (mixed, and FP64 unless PSIB_BFS64=0) reads
                                and writes by its algorithm (polyhedra, tet vertices, fragment records
                                or sums); 0 when every tet was walked depth first */
    long long corrected_items; /* atomic accumulation: tet images walked a second time to add their mass
                                  correction (their FP32 walk missed the exact q-volume by more than 1e-14) */
    int accumulation;        /* 1: fragments were added to per-voxel sums with atomics; 0: sorted records */
} psib_stats;

typedef struct {
    int precision;     /* PSIB_FP64, PSIB_MIXED or PSIB_FP64_CENTRAL */
    int deterministic; /* 0 (default): mixed and FP64-central calls add each fragment's moments to
                          per-voxel sums with FP64 atomics and merge the sums into the fields once (the
                          last bits may differ between runs); 1: fragments are written as records,
                          sorted by voxel and applied in a fixed order (bit-reproducible).  PSIB_FP64
                          always applies the records in the reference's order (bit for bit). */
    int memory;        /* PSIB_HOST or PSIB_DEVICE */
    int device;        /* CUDA device ordinal for PSIB_HOST calls (-1: current) */
    void *stream;      /* cudaStream_t for PSIB_DEVICE calls; NULL: legacy default stream */
    psib_stats *stats; /* optional */
    int refine_mode;   /* PSIB_REFINE_MIDPOINT (0) or PSIB_REFINE_STRETCH */
    double refine_cell[3]; /* stretch: the Lagrangian cell; all <= 0: box / block_dims of a periodic block mesh */
    long long queue_voxels; /* the breadth-first walks (mixed and FP64): tets walked per pass, bounded by the
                               sum of their index-box volumes (the size of every polyhedron queue); 0:
                               automatic (up to 64M, within 35% of the free device memory) */
    int capture;       /* 0: a plain call.  1 (plan): a plain call (mixed precision, deterministic = 0,
                          device memory) that also sizes every buffer for calls like it, with room for
                          25% more tet images, and records their launch plan on this device.
                          2 (capture): such a call with no host synchronisation and no allocation, so
                          that the caller can record it in a CUDA graph and replay it: counts stay on
                          the device, a device-side planner lays out the passes of the walk, and
                          unused passes fall through.  It needs a plan call with the same grids,
                          meshes and fields before it, returns before the work is done and reports
                          failures through psib_capture_status; stats are not filled. */
    int order_cell_bits; /* mixed precision: the tet images of one box volume are walked in the order of a
                            coarse grid of 2^b cells (b bits split over the axes, x first: 7 gives
                            8 x 4 x 4 cells), so that the atomic sums of neighbouring fragments stay in
                            L2; 0: 7, -1: no spatial order, 1..7: b.  capi.autotune_batch picks it. */
} psib_options;

/* Deposit the mesh's tets on the grid: the density branch of psi_voxels
 * (src/cpsi.c:41-112) with refinement as src/refine.c:58-289.
 * refine_max_lvl is capped at 6 like src/refine.c:89-92. */
int psib_voxels(const psib_grid *grid, const psib_mesh *mesh, int mode, double refine_tolerance,
                int refine_max_lvl, const psib_options *opt);

/* A batch of independent deposits -- many cutouts of uneven size, each a
 * psib_voxels call of its own (grids[b], meshes[b]) -- run as one pass: every
 * stage (tessellation, ordering by footprint, the clip walk, the record sort,
 * the field update) is one set of launches over the tets of all cutouts, whose
 * work queues mix them.  Each cutout's fields equal those of its own
 * psib_voxels call (FP64: bit for bit).  The reference has no batch call; it
 * replaces a loop of psi_voxels calls (src/cpsi.c:41).
 * All pointers are device memory (options->memory must be PSIB_DEVICE), every
 * grid has the same set of fields, 1 <= nbatch <= 65535, fewer than 2^32
 * voxels and 2^31 elements in all.  The refinement arguments apply to every
 * cutout. */
int psib_voxels_batch(const psib_grid *grids, const psib_mesh *meshes, int nbatch, int mode,
                      double refine_tolerance, int refine_max_lvl, const psib_options *opt);

/* Adjoint of the density deposit.  The reference has no adjoint; this is
 * the backward pass of psib_voxels's m field for differentiable use.
 *
 * grad->fields[PSIB_M] holds dL/dm per voxel (same grid as the forward call;
 * every other field must be NULL).  The gradient of L with respect to the
 * particle positions is ADDED to grad_pos (npart x 3 doubles) and, when
 * grad_mass is not NULL, the gradient with respect to the element masses to
 * grad_mass (nelem doubles).  grad_vel is accepted for ABI stability and left
 * unchanged: the m field does not depend on the velocities.  The clip is
 * recomputed in FP64 (options->precision is ignored); each fragment's mass
 * fraction is differentiated through the faces it shares with its tet.
 * Gradients are summed with atomics, so the last bits may vary between runs.
 * Elements are refined as psib_voxels refines them (refine_tolerance and
 * refine_max_lvl of the forward call, midpoint criterion): a refined tet vertex
 * passes its gradient to the element's nodes with the trilinear (8-node) or
 * triquadratic (27-node) weights of its place in the element; the refinement
 * decisions are piecewise constant and carry no gradient.
 * Memory and stream follow options as in psib_voxels. */
int psib_voxels_adjoint(const psib_grid *grad, const psib_mesh *mesh, double refine_tolerance,
                        int refine_max_lvl, double *grad_pos, double *grad_vel, double *grad_mass,
                        const psib_options *opt);

/* Adjoint of every grid field.  The reference has no adjoint; this is the
 * backward pass of a psib_voxels deposit into zeroed fields, for differentiable
 * use of all its moments (src/geometry.c:81-186 defines them).
 *
 * fwd holds the fields that deposit produced (m, and any of x, v, xx, xv, vv;
 * a second moment needs its first moments); grad->fields[f] holds dL/d(field f)
 * on the same grid, or NULL for a field L does not depend on (a gradient needs
 * its forward field).  The gradients of L with respect to the particle
 * positions and velocities (npart x 3 doubles each) and the element masses
 * (nelem doubles) are ADDED to grad_pos, grad_vel and grad_mass (the last two
 * may be NULL).  The clip is recomputed in FP64; each fragment's moments are
 * differentiated through the motion of its faces that lie on its tet's faces,
 * the tet's density and the interpolated velocity field.  The reference's
 * pairing of the x-v cross terms with the tet's first vertex
 * (src/geometry.c:137-146) is differentiated as it is.  Gradients are summed with
 * atomics, so the last bits may vary between runs.  Device memory only, on
 * options->stream.  Refinement as in psib_voxels_adjoint. */
int psib_voxels_adjoint_fields(const psib_grid *grad, const psib_grid *fwd, const psib_mesh *mesh,
                               double refine_tolerance, int refine_max_lvl, double *grad_pos, double *grad_vel,
                               double *grad_mass, const psib_options *opt);

/* The status the work of capture-mode calls (options->capture = 2) left on the
 * current device, read after their graph has run (this synchronises the
 * device): PSIB_OK, or the PSIB_ERR_* code of the first failure -- e.g.
 * PSIB_ERR_OVERFLOW when the tet images outgrew the planned buffers.  Clears
 * it.  It has no counterpart in the reference. */
int psib_capture_status(void);

/* Message for the last failure on this thread ("" if none). */
const char *psib_last_error(void);

/* ABI version (PSIB_ABI_VERSION) and the number of visible CUDA devices
 * (0 when none or the driver is absent). */
int psib_abi_version(void);
int psib_device_count(void);

/* Page-locked host memory for grid fields, so that host<->device copies run
 * at full link speed.  Returns NULL on failure (e.g. no device); release with
 * psib_host_free. */
void *psib_host_alloc(unsigned long long bytes);
void psib_host_free(void *p);

/* Release the library's cached device buffers on the current device. */
int psib_release_device_memory(void);

/* Density deposit for callers that must not have the library allocate device
 * memory -- e.g. an application whose own pool allocator owns all of the GPU's
 * memory, or a time-critical loop that cannot afford an allocation.  It has no
 * counterpart in the reference.
 *
 * Adds the mass of ntets tets to grid->fields[PSIB_M] (a device pointer; the
 * other fields must be NULL).  tet_pos is a device array of ntets x 4 x 3
 * doubles (vertex-major, positions already periodic-unwrapped by the caller),
 * tet_mass a device array of ntets doubles (NULL: 1).  The tets are clipped
 * against the grid window and deposited as psib_voxels would deposit simplex
 * elements (same fragments; the sum per voxel may round differently because it
 * is accumulated with atomics).  Runs on `stream` and returns when it is done.
 *
 * It calls no cudaMalloc or cudaFree: its scratch is a fixed array of about
 * 7.9 MiB in device memory, held by every GPU that loads the library until
 * the process exits.  Limit: a tet is too large when the bisection of its
 * voxel index box (clamped to the grid window) is deeper than 12 levels, i.e.
 * when the sum over the three axes of ceil(log2(box size)) exceeds 12 (so
 * 16x16x16 voxels is accepted, 16x16x32 rejected).  A first pass checks every
 * tet: if one is too large the call returns PSIB_ERR_ARG and adds nothing to
 * m.  Any other failure (PSIB_ERR_OVERFLOW, PSIB_ERR_INDEX) is found while
 * depositing, so m then holds part of the call's tets.  All calls on a device
 * share that array: calls that overlap on the GPU race.  Every call looks up
 * the array's address (an allocation-free lookup); the first call on a device
 * also loads the library's kernels there and should come before any stream
 * capture. */
int psib_voxels_density_noalloc(const psib_grid *grid, const double *tet_pos, const double *tet_mass,
                                long long ntets, void *stream);

/* The FMA issue rate of the current device in TFLOP/s (2 flop per FMA):
 * precision PSIB_FP64 for FP64, PSIB_MIXED for FP32.  Eight independent FMA
 * chains per thread on every SM, best of three timed launches.  It has no
 * counterpart in the reference: it measures the denominators of the FP64 and
 * FP32 rooflines of the clip walk.  Allocates and frees one small buffer. */
int psib_measure_fma_peak(int precision, double *tflops);

/* Element queries: for each of nboxes boxes (6 doubles each: lo xyz, hi xyz)
 * the elements whose box touches it (closed intervals) -- PSI.RStarTree(mesh)
 * .query(box) (src/PSI.c:817-862) over the tree of src/rtree.c:48-73, whose
 * elements are those that survive the cull against `window` (after their
 * periodic unwrap, src/cpsi.c:309-341): the periodic box of a periodic mesh,
 * +-1e30 for an open one (src/PSI.c:877-893).  No tree is built: the boxes are
 * tested against every element on the GPU.
 *
 * offsets (nboxes + 1) receives the exclusive offsets of each box's results;
 * with elements == NULL nothing else is written (a size query), else the
 * element indices of box b go to elements[offsets[b] .. offsets[b + 1]) in
 * descending index -- the order of the reference's tree while it is one leaf
 * (at most 32 elements; larger trees return the same set in another order).
 * PSIB_ERR_OVERFLOW when capacity is below the total.  Memory follows
 * options->memory (host by default); device-memory calls run on
 * options->stream and return when the results are written. */
int psib_query_elements(const psib_mesh *mesh, const double window[2][3], const double *boxes, long long nboxes,
                        long long *offsets, int *elements, long long capacity, const psib_options *opt);

/* Phase-space samples of the sheet at each of npoints points (3 doubles each)
 * -- PSI.VDF(mesh, sample_pos, tree, refine_tolerance, refine_max_lvl)
 * (src/PSI.c:1022-1057, src/cpsi.c:177-275) for many points at once.  Every
 * element whose box (over the elements that survive the cull against `window`:
 * a tree's window as psib_query_elements describes it, or, as the reference
 * uses when PSI.VDF is given no tree, the mesh's own box -- zero for an open
 * mesh) contains the point is refined from its vertices as stored, with the
 * absolute tolerance refine_tolerance; each of its tets that contains the
 * point (barycentric coordinates >= 0, nonzero volume, src/geometry.c:335-389)
 * gives one sample: density mass / volume (rho) and the velocity interpolated
 * at the point (vel, 3 doubles).  Samples of point p go to
 * [offsets[p], offsets[p + 1]), in the order element (descending), tet.
 * rho == NULL: offsets only.  PSIB_ERR_OVERFLOW when capacity (samples) is
 * below the total.  Memory and stream as psib_query_elements. */
int psib_sample_vdf(const psib_mesh *mesh, const double window[2][3], const double *points, long long npoints,
                    double refine_tolerance, int refine_max_lvl, long long *offsets, double *rho, double *vel,
                    long long capacity, const psib_options *opt);

/* A persistent element index: what PSI.RStarTree(mesh) builds once and its
 * queries reuse (src/PSI.c:865-896, src/rtree.c:48-73).  psib_index_create
 * copies the mesh to the device, culls its elements against `window`, keeps
 * their boxes and the cell index over them, and returns a handle; the index
 * holds the mesh as it was then.  psib_index_query and psib_index_sample_vdf
 * then answer exactly as psib_query_elements and psib_sample_vdf with the same
 * mesh and window, at the cost of the query alone (no upload, no index build):
 * the form for many small calls, PSI.VDF(mesh, point, tree) in a loop.  Points,
 * boxes and outputs follow options->memory (host by default).  An index lives
 * on the device that was current at its creation until psib_index_destroy. */
typedef struct psib_index psib_index;
int psib_index_create(const psib_mesh *mesh, const double window[2][3], psib_index **index,
                      const psib_options *opt);
int psib_index_query(psib_index *index, const double *boxes, long long nboxes, long long *offsets, int *elements,
                     long long capacity, const psib_options *opt);
int psib_index_sample_vdf(psib_index *index, const double *points, long long npoints, double refine_tolerance,
                          int refine_max_lvl, long long *offsets, double *rho, double *vel, long long capacity,
                          const psib_options *opt);
void psib_index_destroy(psib_index *index);

/* Snapshot readers: a Gadget-2 (format 1) file as the periodic trilinear mesh
 * of PSI.Mesh(loader='gadget2') (src/mesh.c:35-160) or, with 64-bit particle
 * IDs and particles numbered in tiles of 4^3, loader='gevolution'
 * (src/mesh.c:163-302); src/PSI.c:659-709 is the caller they replace.
 *
 * psib_peek_gadget2 reads the header: the number of type-1 particles (also
 * the number of elements) and the box size; the box is [0, box_size]^3.
 * psib_load_* fill pos and vel (npart x 3 doubles, particle p at row ID[p]),
 * mass (npart doubles, each header.mass[1] / npart) and connectivity
 * (npart x 8 ints, elements of 8 nodes); npart must equal the header's count.
 * Host memory only; no device is needed.  A file whose IDs are not a
 * permutation of 0..npart-1 fails with PSIB_ERR_INDEX; one whose particles do
 * not form a cubic lattice (gevolution: of a side that is a multiple of 4),
 * or whose block lengths disagree with npart, with PSIB_ERR_ARG. */
int psib_peek_gadget2(const char *filename, long long *npart, double *box_size);
int psib_load_gadget2(const char *filename, long long npart, double *pos, double *vel, double *mass,
                      int *connectivity);
int psib_load_gevolution(const char *filename, long long npart, double *pos, double *vel, double *mass,
                         int *connectivity);

#ifdef __cplusplus
}
#endif
#endif /* PSI_B200_H */
