// psib_kernels.h -- argument blocks and launchers shared by the translation
// units of libpsi_b200 (host orchestration in pipeline.cu; kernels in
// clip_fp64.cu, clip_mixed.cu, tess.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace psib {

// field presence flags
enum : unsigned { F_X = 1u, F_V = 2u, F_XX = 4u, F_XV = 8u, F_VV = 16u };

// Tet images ("items").  Each image's frame is one contiguous record of
// FRAME doubles -- the 4 vertex positions (vertex-major, periodic image
// applied), the 4 vertex velocities, the tet mass and one pad -- because the
// clip and apply kernels visit images in footprint and voxel order, not in
// index order, and a contiguous frame costs them 7 sectors instead of 25.
// Images are numbered in the reference's visiting order (element,
// refinement path, tet, periodic image).
constexpr int FRAME = 26;
constexpr int FR_U = 12, FR_MASS = 24;
struct ItemArrays {
    double *frame;   // FRAME x cap
    int *elem;       // cap: element index
    int *pid;        // 4 x cap: per vertex the particle id (>= 0), or for a vertex of a refined
                     // element its place in the element, refine_vertex_code (<= -2)
    uint16_t *key;   // cap: footprint key (KEY_DEEP: the deep-tree kernel's; KEY_PAD: no image)
    uint16_t *grid;  // cap: the image's cutout in a batch (null for a single grid)
    long long cap;
};

struct GridDev {
    int n[3];
    double w0[3], w1[3], d[3];
};

// Footprint key of a tet image (ItemArrays.key), sorted ascending to order the
// clip's work: KEY_DEEP for the deep-tree kernel, else the index-box volume
// (1..256: a box the main walk takes has a bisection at most 8 deep) in the
// high bits, larger boxes first, and in the low KEY_CELL_BITS a coarse cell of
// the grid (8 x 4 x 4 cells) holding the box's low corner, so that images of
// one volume are walked in spatial order and their fragments' atomic sums stay
// in L2.  KEY_PAD marks the unused entries of a fixed-size item buffer (the
// capture mode sorts them past every image).
constexpr unsigned KEY_DEEP = 0xFFFEu;
constexpr unsigned KEY_PAD = 0xFFFFu;
constexpr int KEY_CELL_BITS = 7;
// A vertex of a tet of a refined element, as an image's pid entry: its parameter coordinates in
// the element's unit cube in units of 1/128 (0..128 each; a leaf cube of level d has side
// 128 >> d) and the level d (0..6); always <= -2, so never a particle id or the -1 of "none".
__host__ __device__ __forceinline__ int refine_vertex_code(int x, int y, int z, int d)
{
    return -2 - (x | (y << 8) | (z << 16) | (d << 24));
}
__host__ __device__ __forceinline__ void refine_vertex_decode(int pid, int *xyz, int &d)
{
    const int c = -2 - pid;
    xyz[0] = c & 0xFF;
    xyz[1] = (c >> 8) & 0xFF;
    xyz[2] = (c >> 16) & 0xFF;
    d = (c >> 24) & 0x7;
}

__host__ __device__ __forceinline__ long long key_volume(unsigned k)
{
    if (k >= KEY_DEEP) return 1ll << 40;
    const long long v = 256 - (long long)(k >> KEY_CELL_BITS);
    return v > 0 ? v : 1;
}

// Atomic accumulation of central-form fragments (options deterministic == 0,
// mixed and FP64-central): instead of writing a record, each fragment adds its
// mass, first and second moments to per-voxel sums with FP64 atomics (L2), and
// one pass at the end merges the sums into the fields.  sum holds `stride`
// doubles per voxel: [0] mass m; [ox + i] m (x_f - c)_i about the voxel's centre
// c; [ov + i] m (v_f - u)_i about the reference velocity u of the voxel's tile of
// ACC_TILE^3 voxels; [oxx + k] m (S_xx + dx dx^T) over (xx xy xz yy yz zz);
// [oxv + 3i + j] m (S_xv + dx dv^T)_ij; [ovv + k] as oxx.  An offset of -1 marks
// sums not kept.  dx and dv are taken about reference points of the voxel that
// lie close to its means -- the centroids of the first fragment that reaches
// the voxel, which claims them with one 64-bit compare-and-swap (rx, rv; see
// psib_accum.cuh) -- so that the later E[xx] - E[x]E[x] (and vv, xv) does not
// cancel even in voxels made of tiny fragments.  The velocity reference is
// stored relative to the mean velocity of the voxel's tile of ACC_TILE^3 voxels.
constexpr int ACC_TILE = 8;
struct AccArgs {
    double *sum;              // null: write records
    int stride, ox, ov, oxx, oxv, ovv;
    const double *vref;       // 3 per tile
    const long long *toff;    // batch: first tile of each cutout (null: one grid, tiles from 0)
    const double *factor;     // correction pass: per image mass factor (null: 1)
    unsigned long long *rx;   // per voxel: packed position reference (0: not yet claimed)
    unsigned long long *rv;   // per voxel: packed velocity reference (0: not yet claimed)
};

// Tile of voxel (i, j, k) of grid g: ACC_TILE^3 voxels, numbered within the grid.
__host__ __device__ __forceinline__ long long acc_tile(const GridDev &g, int i, int j, int k)
{
    const long long ty = (g.n[1] + ACC_TILE - 1) / ACC_TILE, tz = (g.n[2] + ACC_TILE - 1) / ACC_TILE;
    return ((long long)(i / ACC_TILE) * ty + j / ACC_TILE) * tz + k / ACC_TILE;
}
__host__ __device__ __forceinline__ long long acc_tiles(const GridDev &g)
{
    long long t = 1;
    for (int a = 0; a < 3; ++a) t *= (g.n[a] + ACC_TILE - 1) / ACC_TILE;
    return t;
}

struct MeshDev {
    int elemtype;
    long long npart, nelem;
    const double *pos, *vel, *mass;
    const int *conn;
    int bdim[3];  // particle lattice of an implicit block mesh
    int edim[3];  // element lattice of an implicit block mesh
    int periodic;
    double box0[3], box1[3];
    double ptol2;   // midpoint refinement: squared tolerance (reftol x the grid's smallest cell)^2
    double lag[3];  // stretch refinement: the Lagrangian cell
};

struct ClipArgs {
    ItemArrays it;
    const int *order;        // queue position -> item (may be null: identity)
    long long order_base;    // first queue position of this launch
    long long n;             // queue entries of this launch
    unsigned long long *head;
    // capture mode: the queue entries and first position of the launch read from device memory
    const unsigned long long *n_dev, *base_dev;
    GridDev g;
    int mom_order;           // polynomial order of the moments (0, 1, 2)
    unsigned *status;
    unsigned long long *counters; // fragments, fragment vertices, splits
    // a batch of cutouts: each image's grid is grids[it.grid[t]], its voxels are
    // numbered from voff[it.grid[t]] (null for a single grid: g, from 0)
    const GridDev *grids;
    const unsigned long long *voff;
    // fragment records
    unsigned long long *rec_key; // voxel << rec_ibits | item
    double *rec_mom;             // rec_nmom doubles per record
    unsigned long long *rec_n;
    unsigned long long rec_cap;
    int rec_nmom;
    long long rec_item_base;
    int rec_ibits;           // bits of the item field of a record key
    double *scale;           // FP32 kernel: per item, exact / FP32 q-volume
    void *scratch;           // per-thread scratch regions (grid x block of them)
    // adjoint kernels
    const double *adj_gm;    // dL/dm per voxel
    double *adj_gpos;        // dL/dpos per particle (accumulated)
    long long adj_npart;
    double *adj_gmass;       // dL/dmass per element (accumulated), may be null
    double adj_mass_factor;  // tet mass / element mass of an unrefined element
    const double *adj_coef;  // full adjoint: ADJ_NCOEF coefficients per voxel (null: the m field only, adj_gm)
    double *adj_gvel;        // full adjoint: dL/dvel per particle (accumulated), may be null
    MeshDev adj_mesh;        // the mesh: corner ids and weights of the vertices of refined images
    AccArgs acc;             // atomic accumulation (acc.sum != null) instead of records
};

struct TessArgs {
    MeshDev m;
    GridDev g;
    long long e0, e1;          // element range
    int max_lvl;
    int quad;                  // some element is triquadratic (27 nodes): the kernel variant that holds them
    int refine_mode;           // 0: the reference's midpoint test (m.ptol2); 1: stretch beyond `stretch` x m.lag
    double stretch;
    int cbits[3];              // bits of the footprint key's coarse cell per axis (0 0 0: no spatial order)
    // a batch of cutouts (nbatch > 0): element E belongs to cutout b with
    // eoff[b] <= E < eoff[b + 1]; its mesh and grid are meshes[b], grids[b]
    int nbatch;
    const MeshDev *meshes;
    const GridDev *grids;
    const long long *eoff;
    const long long *offset;   // per element, exclusive (emit)
    long long offset_base;
    int *count;                // per element (count)
    ItemArrays it;
    unsigned *status;
    unsigned long long *counters; // elements kept, tets
};

// ---- launchers (return cudaError_t of the launch) ----
// big: the kernel for images whose bisection tree is deeper than DMAX_MAIN
cudaError_t launch_clip_fp64(const ClipArgs &a, bool big, int grid, int block, cudaStream_t s);
// centroid-form records: the FP32 main kernel (fp64_walk: the FP64 one); big -> the FP64
// deep-tree kernel
cudaError_t launch_clip_mixed(const ClipArgs &a, bool big, bool fp64_walk, int grid, int block, cudaStream_t s);
// bytes of one thread's scratch region
size_t scratch_bytes_fp64(bool big);
size_t scratch_bytes_mixed(bool big, bool fp64_walk);
// resident blocks per SM of a clip kernel at this block size
int clip_blocks_per_sm_fp64(bool big, int block);
int clip_blocks_per_sm_mixed(bool big, bool fp64_walk, int block);
// adjoint of the density deposit (FP64 walk, no records); full: every field, through adj_coef
cudaError_t launch_adjoint(const ClipArgs &a, bool big, int grid, int block, cudaStream_t s);
int adjoint_blocks_per_sm(bool big, int block, bool full = false);

// Per-voxel coefficients of the full adjoint (psib_adjoint.cuh) from the
// forward fields and their upstream gradients (either may be null per field).
struct AdjCoefArgs {
    const double *F[6];      // forward fields m x v xx xv vv
    const double *G[6];      // dL/d(field), null: 0
    double *coef;            // ADJ_NCOEF per voxel
    long long nvox;
};
cudaError_t launch_adj_coeffs(const AdjCoefArgs &a, cudaStream_t s);

// Breadth-first clip of the main tet images (mixed precision, bfs.cu).
// Polyhedra in flight between levels, in 32-wide tiles: element e's vertex v,
// coordinate c at x[((e/32 * MAXV + v) * 3 + c) * 32 + e%32], its links at
// nb[(e/32 * MAXV + v) * 32 + e%32]; nv == 0 marks an element to skip.
struct PolyQueue {
    float *x;
    uint32_t *nb;
    uint8_t *nv;
    uint8_t *win;             // window planes still to cut: bit 2a keeps x_a >= w0_a, 2a+1 keeps x_a <= w1_a
    uint32_t *box;            // 3 per element: lo | hi << 16
    uint32_t *item;
    unsigned long long *count;
    unsigned long long cap;
    // leaf queue: polyhedra of more than BfsArgs::leaf_split vertices are counted here and stored
    // from the end of the buffer (element cap - 1 - j), so that a leaf warp's lanes mostly hold
    // fragments of similar vertex counts; the two ends together stay within cap
    unsigned long long *count_hi;
    // FP64 walk (x null): element e's vertex v holds position then q, c = 0..5, at
    // xq[((e/32 * MAXV + v) * 6 + c) * 32 + e%32]
    double *xq;
};
struct BfsArgs {
    ClipArgs c;               // frames, queue order, grid, records, status, counters, scale
    PolyQueue in, out, leaf;  // level: in -> out and leaf; init: -> out and leaf; leaf kernel: leaf
    const long long *passes;  // init: queue positions of pass p are [passes[p], passes[p + 1])
    unsigned long long *pass_idx; // the current pass (advanced by launch_bfs_advance)
    int *dfs_list;            // init: images that need the window clip (depth-first kernel)
    unsigned long long *dfs_count;
    int last;                 // level: the last level, which must leave no polyhedron unfinished
    double *vsum;             // per image: sum of its fragment q-volumes (leaf), for the mass correction
    unsigned long long *bytes; // algorithmic bytes the walk reads and writes (polyhedra, frames, records)
    int window_bfs;           // init: window-clipped images are walked here too (else listed for the
                              // depth-first kernel)
    int level_blocks;         // level: resident blocks per SM (0: as many as fit)
    int leaf_split;           // level: leaves of more vertices go to the leaf queue's high end (0: none)
    int level_split;          // level: children of more vertices go to the level queue's high end (0: none)
    int fp64;                 // the FP64 walk (bfs_fp64.cu): queues of FP64 positions and q, raw records
};
// each launches one resident wave of grid-stride blocks on num_sms SMs
cudaError_t launch_bfs_init(const BfsArgs &a, int num_sms, cudaStream_t s);
cudaError_t launch_bfs_level(const BfsArgs &a, int num_sms, cudaStream_t s);
cudaError_t launch_bfs_leaf(const BfsArgs &a, int num_sms, cudaStream_t s);
cudaError_t launch_bfs_finalize(const BfsArgs &a, long long nitems, int num_sms, cudaStream_t s);
cudaError_t launch_bfs_advance(const BfsArgs &a, cudaStream_t s);
// the FP64 walk's init, level and leaf kernels (the pass table, finalize and advance are shared)
cudaError_t launch_bfs64_init(const BfsArgs &a, int num_sms, cudaStream_t s);
cudaError_t launch_bfs64_level(const BfsArgs &a, int num_sms, cudaStream_t s);
cudaError_t launch_bfs64_leaf(const BfsArgs &a, int num_sms, cudaStream_t s);
// kernel attributes and occupancy, queried once before any launch or stream capture
void bfs_prepare();
void bfs64_prepare();
// the shared-memory share of the unified L1 of the level kernel, in percent (0: the driver's choice)
void bfs_level_carveout(int percent);

cudaError_t launch_tess_count(const TessArgs &a, cudaStream_t s);
cudaError_t launch_tess_emit(const TessArgs &a, cudaStream_t s);

// Sorted fragment records gathered into key order: voxel, item and moments.
struct GatherArgs {
    const unsigned long long *key; // sorted keys
    const unsigned *perm;          // sorted position -> record
    const double *mom;             // record moments, record order
    long long nrec;
    int nmom, ibits;
    unsigned *vox;                 // out: voxel of each sorted record
    unsigned *item;                // out: item of each sorted record
    double *mom_sorted;            // out: moments in key order (null: not gathered)
};
cudaError_t launch_gather_records(const GatherArgs &a, cudaStream_t s);

// One thread per voxel run of the sorted records.
struct ApplyArgs {
    const unsigned *run_vox;       // voxel of each run
    const int *run_cnt;            // records of each run
    const long long *run_off;      // first sorted record of each run
    long long nruns;
    const unsigned *item;          // item of each sorted record
    const double *mom;             // moments: of each sorted record, or (central) in record order
    const unsigned *perm;          // central: sorted position -> record
    int nmom;
    int central;                   // records hold m0, q-centroid, central second moment
    const double *scale;           // per item mass correction (central records)
    ItemArrays it;
    long long item_base;
    double *M, *X, *V, *XX, *XV, *VV;
    // a batch: voxel v of the runs belongs to cutout b with voff[b] <= v < voff[b + 1],
    // whose fields are fptr[6 b .. 6 b + 5] (m x v xx xv vv); M..VV are then cutout 0's
    int nbatch;
    const unsigned long long *voff;
    double *const *fptr;
};
cudaError_t launch_apply_records(const ApplyArgs &a, cudaStream_t s);

// The atomic accumulation's sums merged into the fields, voxels [v0, v1) of the
// call's voxel numbering (fields and batch tables as in ApplyArgs).
struct FinalArgs {
    ApplyArgs ap;             // fields (M..VV, nbatch, voff, fptr)
    AccArgs acc;
    GridDev g;                // one grid, or
    const GridDev *grids;     // a batch's grids
    long long v0, v1;
};
cudaError_t launch_acc_finalize(const FinalArgs &a, int num_sms, cudaStream_t s);
// Reference velocities of the tiles: the mass-weighted mean velocity of the
// images whose first vertex lies in the tile (0 where none does).  tsum: 4
// doubles per tile, zeroed by the caller.
cudaError_t launch_vref(const ItemArrays &it, long long nitems, const GridDev &g, const GridDev *grids,
                        const AccArgs &acc, double *tsum, long long ntiles, int num_sms, cudaStream_t s,
                        const long long *n_items = nullptr);
// Images whose breadth-first mass correction (scale) differs from 1 by more
// than tol: appended to list (count in *n), with factor[t] = scale[t] - 1 and
// their footprint keys gathered into keys.  n_items (may be null): the number
// of images, read on the device, below nitems.
cudaError_t launch_correction_select(const ItemArrays &it, const double *scale, long long nitems, double tol,
                                     int *list, uint16_t *keys, double *factor, unsigned long long *n,
                                     int num_sms, cudaStream_t s, const long long *n_items = nullptr);

// ---- annihilation mode (annihilation.cu; the element stage in tess.cu) ----
// A tet record: 4 oriented vertices (vertex-major), rho = mass / volume, the
// volume, and the bounding box (lo, hi).
constexpr int TREC = 20;
constexpr int TR_RHO = 12, TR_VOL = 13, TR_BOX = 14;

struct AnnTessArgs {
    MeshDev m;
    GridDev g;
    int max_lvl;
    int quad;
    // count pass: per element the number of tets of each side (0: culled) and the
    // unwrapped element box (6 doubles: lo, hi)
    int *cnt_a, *cnt_b;
    double *ebox;
    // emit pass: exclusive offsets and the tet records; side A is refined from the
    // unwrapped element, side B from the element's vertices as stored
    const long long *off_a, *off_b;
    double *tets_a, *tets_b;
    unsigned *status;
    unsigned long long *counters; // elements kept, side-A tets
};
cudaError_t launch_ann_tess(const AnnTessArgs &a, bool emit, cudaStream_t s);

// Uniform cells over the element boxes: origin, cell size and cells per axis.
struct CellGrid {
    double o[3], h[3];
    long long n[3];
};
struct AnnArgs {
    long long nelem;
    const double *ebox;
    const int *cnt_a, *cnt_b;
    const long long *off_a, *off_b;
    const double *tets_a, *tets_b;
    CellGrid cg;
    // cell registrations: (cell key, element)
    const long long *reg_off; // per element, exclusive (emit)
    long long *reg_cnt;       // per element (count)
    unsigned long long *reg_key;
    int *reg_elem;
    long long nreg;
    const long long *run_lo, *run_hi; // per sorted registration: its cell's run [lo, hi)
    // element pairs: key (e << 32) | (2^32 - 1 - e1), so that sorting gives e ascending, e1 descending
    const long long *pair_off;
    long long *pair_cnt;
    unsigned long long *pair_key;
    long long npair;
    // side-A tet slots of the element pairs: slot u is tet u - aoff[p] of pair p's element e
    const long long *aoff;
    long long nslot, slot0, slot1; // slots [slot0, slot1) of this launch
    const long long *tp_excl; // per slot, exclusive over all slots (emit); tp_base: that of slot0
    long long tp_base;
    long long *tp_cnt;        // per slot (count)
    int2 *tpairs;             // (side-A tet, side-B tet) of every tet pair of the chunk
    uint16_t *tp_key;         // emit: per tet pair, larger voxel boxes of the pair's walk first
    GridDev g;                // the grid (tet-pair keys)
    unsigned *status;
    // queries: sorted unique cell keys of the registrations, their runs
    const unsigned long long *run_key;
    const long long *run_off;
    const int *run_cnt;
    long long nruns;
    // query boxes (6 doubles: lo, hi) or points (3 doubles), their result counts and keys
    // (q << 32) | (2^32 - 1 - e), sorted afterwards: q ascending, e descending
    const double *qry;
    long long nq;
    long long *q_cnt;
    const long long *q_off;
    unsigned long long *q_key;
    unsigned long long *q_n;  // brute-force query: emission counter
};
// stats of the kept element boxes: 2 x 3 ordered-int min/max, 3 extent sums, kept count
cudaError_t launch_ann_box_stats(const AnnArgs &a, unsigned long long *out, double *ext, cudaStream_t s);
cudaError_t launch_ann_cells(const AnnArgs &a, bool emit, cudaStream_t s);
cudaError_t launch_ann_runs(const unsigned *run_cnt_u, const long long *run_off, long long nruns, long long *lo,
                            long long *hi, cudaStream_t s);
cudaError_t launch_ann_pairs(const AnnArgs &a, bool emit, cudaStream_t s);
cudaError_t launch_ann_pair_sides(const AnnArgs &a, long long *na, cudaStream_t s);
cudaError_t launch_ann_tpairs(const AnnArgs &a, bool emit, cudaStream_t s);
// chunk plan: bounds[k] = the first slot whose exclusive tet-pair offset reaches k * budget
// (bounds[0] = 0, bounds[nb] = nslot); tp_excl holds nslot + 1 offsets
cudaError_t launch_ann_chunk_bounds(const long long *tp_excl, long long nslot, long long budget, int nb,
                                    long long *bounds, cudaStream_t s);

// The cell of coordinate x on axis i (clamped to the grid; NaN to cell 0), and
// the run of the sorted registrations whose cell key is k (-1: none).
__device__ __forceinline__ long long cell_of(const CellGrid &cg, int i, double x)
{
    double f = floor((x - cg.o[i]) / cg.h[i]);
    if (!(f >= 0.0)) f = 0.0;
    return f < (double)cg.n[i] ? (long long)f : cg.n[i] - 1;
}
__device__ __forceinline__ unsigned long long point_cell(const CellGrid &cg, const double *s)
{
    return (unsigned long long)((cell_of(cg, 0, s[0]) * cg.n[1] + cell_of(cg, 1, s[1])) * cg.n[2] + cell_of(cg, 2, s[2]));
}
__device__ __forceinline__ long long find_run(const AnnArgs &a, unsigned long long k)
{
    long long lo = 0, hi = a.nruns;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (a.run_key[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    return (lo < a.nruns && a.run_key[lo] == k) ? lo : -1;
}

// the element boxes of a query: cull against a.g's window, kept flag in cnt_a and cnt_b
cudaError_t launch_elem_boxes(const AnnTessArgs &a, cudaStream_t s);
// box queries, every (box, element) pair tested (count: q_cnt; emit: q_key via q_n)
cudaError_t launch_query_boxes(const AnnArgs &a, bool emit, cudaStream_t s);
// point queries through the cell index (count: q_cnt; emit: q_key at q_off)
cudaError_t launch_query_points(const AnnArgs &a, bool emit, cudaStream_t s);

// Phase-space samples of (point, element) pairs (psi_sample_vdf, src/cpsi.c:177-275).
struct VdfArgs {
    MeshDev m;                // ptol2 = refine_tolerance^2
    int max_lvl, quad;
    const double *points;
    const unsigned long long *pairs; // sorted keys (point << 32) | (2^32 - 1 - element)
    long long npair;
    long long *cnt;           // count: samples per pair
    const long long *off;     // emit: exclusive sample offset per pair
    double *rho, *vel;
    unsigned *status;
};
cudaError_t launch_vdf_samples(const VdfArgs &a, bool emit, cudaStream_t s);
// One point (a.points[0]) through the cell index x on one thread: its samples, in the order
// of the pairs above, written while fewer than cap; their number to *count.
cudaError_t launch_vdf_point(const VdfArgs &a, const AnnArgs &x, unsigned long long *count, long long cap,
                             cudaStream_t s);
// out[i] = the element of sorted query key i
cudaError_t launch_keys_elem(const unsigned long long *keys, long long n, int *out, cudaStream_t s);
// out[p] = pair_soff[q_off[p]] for p in [0, np]: each point's first sample
cudaError_t launch_gather_ll(const long long *src, const long long *idx, long long n, long long *out, cudaStream_t s);

struct AnnClipArgs {
    const int2 *tpairs;
    long long n;             // tet pairs of this launch
    const int *list;         // null: tet pairs [0, n); else their indices
    const double *tets_a, *tets_b;
    GridDev g;
    unsigned long long *head;
    int *deep;               // main kernel: tet pairs whose bisection is deeper than it serves
    unsigned long long *ndeep;
    unsigned long long *rec_key; // voxel << rec_ibits | tet pair
    double *rec_val;
    unsigned long long *rec_n, rec_cap;
    int rec_ibits;
    unsigned *status;
    unsigned long long *counters; // fragments, fragment vertices, splits
    void *scratch;
};
cudaError_t launch_ann_clip(const AnnClipArgs &a, bool big, int grid, int block, cudaStream_t s);
size_t ann_scratch_bytes(bool big);
int ann_blocks_per_sm(bool big, int block);
// sequential sum of each voxel run of the sorted records into m
cudaError_t launch_ann_apply(const ApplyArgs &a, cudaStream_t s);

// Record `msg` as this thread's last error (psib_last_error) and return `code`.
int report_error(int code, const char *msg);

} // namespace psib
