// annihilation.cu -- annihilation mode: every pair of tets whose regions
// overlap deposits rho_0 rho_1 x (the volume of their intersection in each
// voxel) into m (src/cpsi.c:115-158, src/geometry.c:226-252).
//
// The reference finds overlapping elements with an R*-tree query per element
// and walks each pair's tets on one CPU thread.  Here the search is a uniform
// grid over the element boxes (sort-based, no tree): every element registers in
// the cells its box covers, and each touching pair (e, e1) is reported once, by
// the cell that holds the low corner of the two boxes' intersection.  The pairs
// are sorted into the reference's order (e ascending, e1 descending: the order
// in which its R*-tree returns them while it is a single leaf), expanded into
// tet pairs whose boxes overlap with positive extent, and each tet pair is
// clipped by one thread: the tet of e cut by the four face planes of the tet of
// e1, then by the window and into voxels by the same bisection as the density
// path.  Each voxel fragment becomes a record (voxel, tet pair); the records
// are sorted and each voxel's run is summed into m in that order.
//
// Built with --fmad=false: the face planes, the clip and the moments repeat the
// reference's double-precision operations.
#include "psib_clip.cuh"

#include <cstdlib>

namespace psib {

// The polyhedron of a tet pair: the intersection of two tets, the window and a
// voxel has up to 14 faces, so 24 vertices when no more than three planes meet
// at a point, and more where the vertex graph repeats a point at which several
// planes meet (tets that share faces, a tet against itself).  The reference's
// buffer holds 64 (include/geometry.h:23).
constexpr int MAXV_ANN = 62;
struct PolyA {
    using real = double;
    using mask_t = uint64_t;
    static constexpr bool has_q = true;
    static constexpr int CAP = MAXV_ANN;
    double x[MAXV_ANN][3];
    double q[MAXV_ANN][3];
    uint32_t nb[MAXV_ANN];
    int nv;
    int lo[3], hi[3];
};

template <int NS>
__host__ __device__ constexpr size_t ann_region_bytes() { return round16(sizeof(PolyA) * NS); }

// ---- element boxes: range and mean extent of the kept ones ----

__device__ __forceinline__ unsigned long long ord_of(double x)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__global__ void k_ann_box_stats(AnnArgs a, unsigned long long* out, double* ext)
{
    unsigned long long mn[3] = {~0ull, ~0ull, ~0ull}, mx[3] = {0ull, 0ull, 0ull};
    double sum[3] = {0.0, 0.0, 0.0};
    unsigned long long kept = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < a.nelem; e += stride) {
        if (a.cnt_a[e] <= 0 && a.cnt_b[e] <= 0) continue;
        kept++;
        for (int i = 0; i < 3; ++i) {
            const double lo = a.ebox[6 * e + i], hi = a.ebox[6 * e + 3 + i];
            const unsigned long long ol = ord_of(lo), oh = ord_of(hi);
            mn[i] = ol < mn[i] ? ol : mn[i];
            mx[i] = oh > mx[i] ? oh : mx[i];
            sum[i] += hi - lo;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        for (int i = 0; i < 3; ++i) {
            const unsigned long long a1 = __shfl_down_sync(0xFFFFFFFFu, mn[i], off);
            const unsigned long long a2 = __shfl_down_sync(0xFFFFFFFFu, mx[i], off);
            mn[i] = a1 < mn[i] ? a1 : mn[i];
            mx[i] = a2 > mx[i] ? a2 : mx[i];
            sum[i] += __shfl_down_sync(0xFFFFFFFFu, sum[i], off);
        }
        kept += __shfl_down_sync(0xFFFFFFFFu, kept, off);
    }
    if ((threadIdx.x & 31) == 0 && kept) {
        for (int i = 0; i < 3; ++i) {
            atomicMin(&out[i], mn[i]);
            atomicMax(&out[3 + i], mx[i]);
            atomicAdd(&ext[i], sum[i]);
        }
        atomicAdd(&out[6], kept);
    }
}

static int grid_for(long long n, int block)
{
    long long b = (n + block - 1) / block;
    return (int)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

cudaError_t launch_ann_box_stats(const AnnArgs& a, unsigned long long* out, double* ext, cudaStream_t s)
{
    k_ann_box_stats<<<grid_for(a.nelem, 256), 256, 0, s>>>(a, out, ext);
    return cudaGetLastError();
}

// ---- cells ----

__device__ __forceinline__ bool kept_elem(const AnnArgs& a, long long e) { return a.cnt_a[e] > 0 || a.cnt_b[e] > 0; }

template <bool EMIT>
__global__ void k_ann_cells(AnnArgs a)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < a.nelem; e += stride) {
        if (!kept_elem(a, e)) {
            if (!EMIT) a.reg_cnt[e] = 0;
            continue;
        }
        long long c0[3], c1[3];
        for (int i = 0; i < 3; ++i) {
            c0[i] = cell_of(a.cg, i, a.ebox[6 * e + i]);
            c1[i] = cell_of(a.cg, i, a.ebox[6 * e + 3 + i]);
        }
        if (!EMIT) {
            a.reg_cnt[e] = (c1[0] - c0[0] + 1) * (c1[1] - c0[1] + 1) * (c1[2] - c0[2] + 1);
            continue;
        }
        long long r = a.reg_off[e];
        for (long long x = c0[0]; x <= c1[0]; ++x)
            for (long long y = c0[1]; y <= c1[1]; ++y)
                for (long long z = c0[2]; z <= c1[2]; ++z) {
                    a.reg_key[r] = (unsigned long long)((x * a.cg.n[1] + y) * a.cg.n[2] + z);
                    a.reg_elem[r] = (int)e;
                    ++r;
                }
    }
}

cudaError_t launch_ann_cells(const AnnArgs& a, bool emit, cudaStream_t s)
{
    if (emit) k_ann_cells<true><<<grid_for(a.nelem, 128), 128, 0, s>>>(a);
    else k_ann_cells<false><<<grid_for(a.nelem, 128), 128, 0, s>>>(a);
    return cudaGetLastError();
}

__global__ void k_ann_runs(const unsigned* cnt, const long long* off, long long nruns, long long* lo, long long* hi)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nruns; r += stride) {
        const long long b = off[r], e = b + cnt[r];
        for (long long i = b; i < e; ++i) {
            lo[i] = b;
            hi[i] = e;
        }
    }
}

cudaError_t launch_ann_runs(const unsigned* run_cnt_u, const long long* run_off, long long nruns, long long* lo,
                            long long* hi, cudaStream_t s)
{
    k_ann_runs<<<grid_for(nruns, 256), 256, 0, s>>>(run_cnt_u, run_off, nruns, lo, hi);
    return cudaGetLastError();
}

// Element pairs: registration i (element e in cell k) against every
// registration of the same cell.  The pair (e, e1) -- e1 == e included, as
// the reference's query of e's own box returns e -- is taken when the boxes
// touch (closed intervals, the query test of src/rtree.c:108-111) and k is
// the cell of the low corner of their intersection, which both boxes cover.
template <bool EMIT>
__global__ void k_ann_pairs(AnnArgs a)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.nreg; i += stride) {
        const int e = a.reg_elem[i];
        const unsigned long long k = a.reg_key[i];
        double lo[3], hi[3];
        for (int c = 0; c < 3; ++c) {
            lo[c] = a.ebox[6 * (long long)e + c];
            hi[c] = a.ebox[6 * (long long)e + 3 + c];
        }
        long long n = 0, w = EMIT ? a.pair_off[i] : 0;
        for (long long j = a.run_lo[i]; j < a.run_hi[i]; ++j) {
            const int e1 = a.reg_elem[j];
            bool touch = true;
            double m[3];
            for (int c = 0; c < 3; ++c) {
                const double l1 = a.ebox[6 * (long long)e1 + c], h1 = a.ebox[6 * (long long)e1 + 3 + c];
                if (hi[c] < l1 || lo[c] > h1) touch = false;
                m[c] = lo[c] > l1 ? lo[c] : l1;
            }
            if (!touch) continue;
            const unsigned long long km =
                (unsigned long long)((cell_of(a.cg, 0, m[0]) * a.cg.n[1] + cell_of(a.cg, 1, m[1])) * a.cg.n[2] +
                                     cell_of(a.cg, 2, m[2]));
            if (km != k) continue;
            if (EMIT) a.pair_key[w++] = ((unsigned long long)e << 32) | (0xFFFFFFFFull - (unsigned long long)e1);
            n++;
        }
        if (!EMIT) a.pair_cnt[i] = n;
    }
}

cudaError_t launch_ann_pairs(const AnnArgs& a, bool emit, cudaStream_t s)
{
    if (emit) k_ann_pairs<true><<<grid_for(a.nreg, 128), 128, 0, s>>>(a);
    else k_ann_pairs<false><<<grid_for(a.nreg, 128), 128, 0, s>>>(a);
    return cudaGetLastError();
}

__device__ __forceinline__ void pair_elems(unsigned long long key, long long& e, long long& e1)
{
    e = (long long)(key >> 32);
    e1 = (long long)(0xFFFFFFFFull - (key & 0xFFFFFFFFull));
}

__global__ void k_ann_pair_sides(AnnArgs a, long long* na)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < a.npair; p += stride) {
        long long e, e1;
        pair_elems(a.pair_key[p], e, e1);
        na[p] = a.cnt_a[e];
    }
}

cudaError_t launch_ann_pair_sides(const AnnArgs& a, long long* na, cudaStream_t s)
{
    k_ann_pair_sides<<<grid_for(a.npair, 256), 256, 0, s>>>(a, na);
    return cudaGetLastError();
}

// Ordering key of a tet pair: the voxel index box of its walk (the two boxes'
// intersection within the window, as the clip computes it), larger boxes
// first.  The clip kernel takes tet pairs in this order so that the 32 lanes
// of a warp walk trees of similar size; the records carry the tet pair's
// index, so the order changes no result.
__device__ __forceinline__ uint16_t walk_key(const GridDev& g, const double* b0, const double* b1)
{
    long long vol = 1;
    for (int c = 0; c < 3; ++c) {
        double cmin = fmax(b0[c], b1[c]), cmax = fmin(b0[3 + c], b1[3 + c]);
        if (g.w0[c] > cmin) cmin = g.w0[c];
        if (g.w1[c] < cmax) cmax = g.w1[c];
        int lo = (int)floor((cmin - g.w0[c]) / g.d[c]);
        int hi = (int)ceil((cmax - g.w0[c]) / g.d[c]);
        if (lo < 0) lo = 0;
        if (hi > g.n[c]) hi = g.n[c];
        const int sz = hi - lo;
        if (vol < 0xFFFF) vol *= (sz > 1 ? sz : 1);
    }
    return (uint16_t)(0xFFFF - (vol < 0xFFFE ? vol : 0xFFFE));
}

// Tet pairs: slot u is side-A tet t of element pair p (u = aoff[p] + t); it
// pairs with every side-B tet of e1 whose box overlaps its own with positive
// extent on every axis (psi_aabb_ixn, src/cpsi.c:293-306).  Slots are taken
// in order and each slot's partners in order, so the tet pairs come in the
// reference's order (e, e1, t, t1).
template <bool EMIT>
__global__ void k_ann_tpairs(AnnArgs a)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long u = a.slot0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; u < a.slot1; u += stride) {
        // the pair p with aoff[p] <= u < aoff[p + 1]
        long long lo = 0, hi = a.npair;
        while (hi - lo > 1) {
            const long long mid = (lo + hi) >> 1;
            if (a.aoff[mid] <= u) lo = mid;
            else hi = mid;
        }
        long long e, e1;
        pair_elems(a.pair_key[lo], e, e1);
        const long long ta = a.off_a[e] + (u - a.aoff[lo]);
        const double* ra = a.tets_a + ta * TREC;
        double b0[6];
        for (int c = 0; c < 6; ++c) b0[c] = ra[TR_BOX + c];
        const long long tb0 = a.off_b[e1], nb = a.cnt_b[e1];
        long long n = 0, w = EMIT ? a.tp_excl[u] - a.tp_base : 0;
        for (long long t1 = 0; t1 < nb; ++t1) {
            const double* rb = a.tets_b + (tb0 + t1) * TREC;
            bool ok = true;
            for (int c = 0; c < 3; ++c) {
                const double l = fmax(b0[c], rb[TR_BOX + c]);
                const double h = fmin(b0[3 + c], rb[TR_BOX + 3 + c]);
                ok = ok && (h > l);
            }
            if (!ok) continue;
            if (EMIT) {
                a.tp_key[w] = walk_key(a.g, b0, rb + TR_BOX);
                a.tpairs[w++] = make_int2((int)ta, (int)(tb0 + t1));
            }
            n++;
        }
        if (!EMIT) a.tp_cnt[u] = n;
    }
}

cudaError_t launch_ann_tpairs(const AnnArgs& a, bool emit, cudaStream_t s)
{
    const long long n = a.slot1 - a.slot0;
    if (emit) k_ann_tpairs<true><<<grid_for(n, 128), 128, 0, s>>>(a);
    else k_ann_tpairs<false><<<grid_for(n, 128), 128, 0, s>>>(a);
    return cudaGetLastError();
}

__global__ void k_ann_chunk_bounds(const long long* excl, long long nslot, long long budget, int nb, long long* bounds)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > nb) return;
    if (k == 0) { bounds[0] = 0; return; }
    if (k == nb) { bounds[nb] = nslot; return; }
    // the first slot u whose exclusive offset excl[u] is >= k * budget
    const long long want = (long long)k * budget;
    long long lo = 0, hi = nslot;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (excl[mid] >= want) hi = mid;
        else lo = mid + 1;
    }
    bounds[k] = lo;
}

cudaError_t launch_ann_chunk_bounds(const long long* tp_excl, long long nslot, long long budget, int nb,
                                    long long* bounds, cudaStream_t s)
{
    k_ann_chunk_bounds<<<(nb + 1 + 127) / 128, 128, 0, s>>>(tp_excl, nslot, budget, nb, bounds);
    return cudaGetLastError();
}

// ---- queries (PSI.RStarTree.query, PSI.VDF) ----

// Every (box, element) pair: the closed-interval test of the reference's
// query (src/rtree.c:108-111) against each kept element's box.
template <bool EMIT>
__global__ void k_query_boxes(AnnArgs a)
{
    const long long total = a.nq * a.nelem;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += stride) {
        const long long q = i / a.nelem, e = i % a.nelem;
        if (!kept_elem(a, e)) continue;
        const double* b = a.qry + 6 * q;
        bool touch = true;
        for (int c = 0; c < 3; ++c)
            if (b[3 + c] < a.ebox[6 * e + c] || b[c] > a.ebox[6 * e + 3 + c]) touch = false;
        if (!touch) continue;
        if (EMIT) {
            const unsigned long long w = atomicAdd(a.q_n, 1ull);
            a.q_key[w] = ((unsigned long long)q << 32) | (0xFFFFFFFFull - (unsigned long long)e);
        } else {
            atomicAdd((unsigned long long*)&a.q_cnt[q], 1ull);
        }
    }
}

cudaError_t launch_query_boxes(const AnnArgs& a, bool emit, cudaStream_t s)
{
    if (emit) k_query_boxes<true><<<grid_for(a.nq * a.nelem, 256), 256, 0, s>>>(a);
    else k_query_boxes<false><<<grid_for(a.nq * a.nelem, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

// A point against the elements registered in its cell: every element whose
// box contains the point (the degenerate query box of src/cpsi.c:212-216)
// is registered there.  A run lists its elements in ascending order; it is
// walked backwards, so each point's pairs come out in descending element
// order -- the keys are written already sorted.
template <bool EMIT>
__global__ void k_query_points(AnnArgs a)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < a.nq; q += stride) {
        const double* s = a.qry + 3 * q;
        const long long r = find_run(a, point_cell(a.cg, s));
        long long n = 0, w = EMIT ? a.q_off[q] : 0;
        if (r >= 0) {
            for (long long j = a.run_off[r] + a.run_cnt[r] - 1; j >= a.run_off[r]; --j) {
                const long long e = a.reg_elem[j];
                bool in = true;
                for (int c = 0; c < 3; ++c)
                    if (s[c] < a.ebox[6 * e + c] || s[c] > a.ebox[6 * e + 3 + c]) in = false;
                if (!in) continue;
                if (EMIT) a.q_key[w++] = ((unsigned long long)q << 32) | (0xFFFFFFFFull - (unsigned long long)e);
                n++;
            }
        }
        if (!EMIT) a.q_cnt[q] = n;
    }
}

cudaError_t launch_query_points(const AnnArgs& a, bool emit, cudaStream_t s)
{
    if (emit) k_query_points<true><<<grid_for(a.nq, 128), 128, 0, s>>>(a);
    else k_query_points<false><<<grid_for(a.nq, 128), 128, 0, s>>>(a);
    return cudaGetLastError();
}

__global__ void k_keys_elem(const unsigned long long* keys, long long n, int* out)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = (int)(0xFFFFFFFFull - (keys[i] & 0xFFFFFFFFull));
}

cudaError_t launch_keys_elem(const unsigned long long* keys, long long n, int* out, cudaStream_t s)
{
    k_keys_elem<<<grid_for(n, 256), 256, 0, s>>>(keys, n, out);
    return cudaGetLastError();
}

__global__ void k_gather_ll(const long long* src, const long long* idx, long long n, long long* out)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) out[i] = src[idx[i]];
}

cudaError_t launch_gather_ll(const long long* src, const long long* idx, long long n, long long* out, cudaStream_t s)
{
    k_gather_ll<<<grid_for(n, 256), 256, 0, s>>>(src, idx, n, out);
    return cudaGetLastError();
}

// ---- the clip of one tet pair ----

// Face plane n.x + d >= 0 of a tet (src/geometry.c:503-558): n = A x B with
// the edge vectors A = a1 - a0, B = b1 - b0 the reference takes for that face
// (the same products and differences up to exact sign changes), d = -n . c
// with c a third of the sum of the face's vertices f0 + f1 + f2.
__device__ __forceinline__ void face_plane(const double* a0, const double* a1, const double* b0, const double* b1,
                                           const double* f0, const double* f1, const double* f2, double* n,
                                           double& d)
{
    double A[3], B[3], c[3];
    for (int i = 0; i < 3; ++i) {
        A[i] = a1[i] - a0[i];
        B[i] = b1[i] - b0[i];
        c[i] = (1.0 / 3.0) * (f0[i] + f1[i] + f2[i]);
    }
    n[0] = A[1] * B[2] - A[2] * B[1];
    n[1] = A[2] * B[0] - A[0] * B[2];
    n[2] = A[0] * B[1] - A[1] * B[0];
    d = -(n[0] * c[0] + n[1] * c[1] + n[2] * c[2]);
}

struct AnnTally {
    unsigned long long frags = 0, verts = 0, splits = 0;
};

__device__ __forceinline__ void ann_write(const AnnClipArgs& a, unsigned long long gi, long long k, double val,
                                           unsigned& st)
{
    const unsigned act = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(act) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(a.rec_n, (unsigned long long)__popc(act));
    base = __shfl_sync(act, base, leader);
    const unsigned long long r = base + __popc(act & ((1u << lane) - 1u));
    if (r < a.rec_cap) {
        a.rec_key[r] = (gi << a.rec_ibits) | (unsigned long long)k;
        a.rec_val[r] = val;
    } else {
        st |= ST_RECORDS;
    }
}

// Tet pair k: psi_voxelize_annihilation (src/geometry.c:226-252) with the
// voxel walk of psi_voxels_init / psi_voxels_next (:806-896) over the
// intersection of the two tets' boxes.  Returns false (and leaves the pair to
// the deep kernel) when its bisection needs more than DMAX slots deep.
template <int NS>
__device__ bool ann_clip_pair(const AnnClipArgs& a, long long k, PolyA* S, unsigned& st, AnnTally& tally,
                              int dmax_allowed)
{
    const GridDev& g = a.g;
    const int2 tp = a.tpairs[k];
    const double* r0 = a.tets_a + (long long)tp.x * TREC;
    const double* r1 = a.tets_b + (long long)tp.y * TREC;
    double p0[4][3], p1[4][3];
    for (int v = 0; v < 4; ++v)
        for (int i = 0; i < 3; ++i) {
            p0[v][i] = r0[3 * v + i];
            p1[v][i] = r1[3 * v + i];
        }
    // window planes and index box of the boxes' intersection (src/geometry.c:816-842)
    int pax[6], psg[6], npl = 0;
    double pdd[6];
    int lo[3], hi[3], depth = 0;
    for (int i = 0; i < 3; ++i) {
        double cmin = fmax(r0[TR_BOX + i], r1[TR_BOX + i]), cmax = fmin(r0[TR_BOX + 3 + i], r1[TR_BOX + 3 + i]);
        const bool clo = g.w0[i] > cmin, chi = g.w1[i] < cmax;
        if (clo) cmin = g.w0[i];
        if (chi) cmax = g.w1[i];
        if (clo) { pax[npl] = i; psg[npl] = 1; pdd[npl] = -cmin; npl++; }
        if (chi) { pax[npl] = i; psg[npl] = -1; pdd[npl] = cmax; npl++; }
        lo[i] = (int)floor((cmin - g.w0[i]) / g.d[i]);
        hi[i] = (int)ceil((cmax - g.w0[i]) / g.d[i]);
        if (lo[i] < 0) lo[i] = 0;
        if (hi[i] > g.n[i]) hi[i] = g.n[i];
        const int sz = hi[i] - lo[i];
        if (sz > 1) depth += 32 - __clz(sz - 1);
    }
    if (depth > dmax_allowed) return false;

    uint64_t freem = (NS >= 64) ? ~0ull : ((1ull << NS) - 1ull);
    int8_t stk[NS];
    int top = 0;
#define PSIB_ALLOC(dst)                                            \
    {                                                              \
        const int _i = __ffsll((long long)freem) - 1;              \
        if (_i < 0) { st |= ST_OVERFLOW; return true; }            \
        freem &= ~(1ull << _i);                                    \
        dst = _i;                                                  \
    }
#define PSIB_FREE(i) (freem |= 1ull << (i))
    int c;
    PSIB_ALLOC(c);
    init_tet(S[c], p0);
    double s[MAXV_ANN];
    // the four faces of the second tet (psi_tet_faces_from_verts), then the window
    double fn[4][3], fd[4];
    face_plane(p1[1], p1[3], p1[1], p1[2], p1[1], p1[2], p1[3], fn[0], fd[0]);
    face_plane(p1[0], p1[2], p1[2], p1[3], p1[2], p1[3], p1[0], fn[1], fd[1]);
    face_plane(p1[3], p1[1], p1[3], p1[0], p1[3], p1[0], p1[1], fn[2], fd[2]);
    face_plane(p1[2], p1[0], p1[0], p1[1], p1[0], p1[1], p1[2], fn[3], fd[3]);
    for (int pl = 0; pl < 4 + npl && S[c].nv > 0; ++pl) {
        PolyA& P = S[c];
        double n[3], dd;
        if (pl < 4) {
            for (int i = 0; i < 3; ++i) n[i] = fn[pl][i];
            dd = fd[pl];
        } else {
            const int w = pl - 4;
            for (int i = 0; i < 3; ++i) n[i] = i == pax[w] ? (double)psg[w] : 0.0;
            dd = pdd[w];
        }
        double smin = 1.0e30, smax = -1.0e30;
        uint64_t um = 0;
        for (int v = 0; v < P.nv; ++v) {
            // ((d + x0 n0) + x1 n1) + x2 n2 (src/geometry.c:418-425)
            double t0 = dd;
            for (int i = 0; i < 3; ++i) t0 += P.x[v][i] * n[i];
            s[v] = t0;
            if (t0 < smin) smin = t0;
            if (t0 > smax) smax = t0;
            if (t0 < 0.0) um |= 1ull << v;
        }
        if (smin >= 0.0) continue;
        if (smax <= 0.0) { P.nv = 0; break; }
        int o;
        PSIB_ALLOC(o);
        const unsigned e = cut_any<PolyA, false>(P, s, um, S[o], S[o], 0u);
        PSIB_FREE(c);
        c = o;
        if (e) { st |= e; return true; }
    }
    for (int i = 0; i < 3; ++i) { S[c].lo[i] = lo[i]; S[c].hi[i] = hi[i]; }

    const double w = r0[TR_RHO] * r1[TR_RHO] * r0[TR_VOL];
    double mom[10];
    for (;;) {
        PolyA& P = S[c];
        bool done_node = true;
        if (P.nv > 0) {
            int dm = 0, ax = 0;
            for (int i = 0; i < 3; ++i) {
                const int sz = P.hi[i] - P.lo[i];
                if (sz > dm) { dm = sz; ax = i; }
            }
            if (dm <= 1) {
                const unsigned e = reduce_poly(P, mom, 0);
                if (e) { st |= e; return true; }
                if (mom[0] > 0.0) {
                    if (P.lo[0] >= g.n[0] || P.lo[1] >= g.n[1] || P.lo[2] >= g.n[2]) {
                        st |= ST_INDEX;
                    } else {
                        const unsigned long long gi =
                            ((unsigned long long)g.n[1] * P.lo[0] + P.lo[1]) * g.n[2] + P.lo[2];
                        tally.frags++;
                        tally.verts += P.nv;
                        ann_write(a, gi, k, w * mom[0], st);
                    }
                }
            } else {
                tally.splits++;
                const double coord = g.d[ax] * (P.lo[ax] + dm / 2) + g.w0[ax];
                uint64_t um = 0;
                for (int v = 0; v < P.nv; ++v) {
                    s[v] = coord - P.x[v][ax];
                    if (s[v] < 0.0) um |= 1ull << v;
                }
                const int nlo = dm / 2, nup = dm - dm / 2;
                if (um == 0) {
                    P.hi[ax] -= nup;
                    done_node = false;
                } else if (um == (1ull << P.nv) - 1ull) {
                    P.lo[ax] += nlo;
                    done_node = false;
                } else {
                    int l, r;
                    PSIB_ALLOC(l);
                    PSIB_ALLOC(r);
                    const unsigned e = cut_any<PolyA, true>(P, s, um, S[l], S[r], 0u);
                    if (e) { st |= e; return true; }
                    for (int i = 0; i < 3; ++i) {
                        S[l].lo[i] = P.lo[i]; S[l].hi[i] = P.hi[i];
                        S[r].lo[i] = P.lo[i]; S[r].hi[i] = P.hi[i];
                    }
                    S[l].hi[ax] -= nup;
                    S[r].lo[ax] += nlo;
                    PSIB_FREE(c);
                    if (top >= NS) { st |= ST_OVERFLOW; return true; }
                    stk[top++] = (int8_t)l;
                    c = r;
                    continue;
                }
            }
        }
        if (!done_node) continue;
        PSIB_FREE(c);
        if (top == 0) break;
        c = stk[--top];
    }
#undef PSIB_ALLOC
#undef PSIB_FREE
    return true;
}

template <int NS, bool BIG>
__device__ __forceinline__ void ann_clip_loop(const AnnClipArgs& a)
{
    const int lane = threadIdx.x & 31;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    PolyA* S = (PolyA*)((char*)a.scratch + tid * ann_region_bytes<NS>());
    unsigned st = 0;
    AnnTally tally;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(a.head, 32ull);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= (unsigned long long)a.n) break;
        const long long i = (long long)base + lane;
        if (i < a.n) {
            const long long k = a.list ? (long long)a.list[i] : i;
            const bool done = ann_clip_pair<NS>(a, k, S, st, tally, BIG ? DMAX_BIG : DMAX_MAIN);
            if (!done) {
                if (BIG) {
                    st |= ST_DEPTH;
                } else {
                    const unsigned long long d = atomicAdd(a.ndeep, 1ull);
                    a.deep[d] = (int)k;
                }
            }
        }
    }
    if (st) atomicOr(a.status, st);
    if (a.counters) {
        atomicAdd(&a.counters[0], tally.frags);
        atomicAdd(&a.counters[1], tally.verts);
        atomicAdd(&a.counters[2], tally.splits);
    }
}

// Main kernel variants by the minimum number of resident 128-thread blocks per
// SM the register allocation must allow (0: no cap); PSIB_ANN_MINB picks one.
// Measured at 64^3 -> 128^3: 96 registers (no cap) 201 M tet pairs/s, 80
// (6 blocks) 216 M/s, 64 (8 blocks, a few spills) 227 M/s.
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_ann_clip_b(AnnClipArgs a) { ann_clip_loop<NS_MAIN, false>(a); }
__global__ void __launch_bounds__(128) k_ann_clip(AnnClipArgs a) { ann_clip_loop<NS_MAIN, false>(a); }
__global__ void __launch_bounds__(64) k_ann_clip_big(AnnClipArgs a) { ann_clip_loop<NS_BIG, true>(a); }

constexpr int DEFAULT_MINB_ANN = 8;

template <class F>
static auto ann_variant(F&& f)
{
    const char* v = getenv("PSIB_ANN_MINB");
    switch (v && *v ? atoi(v) : DEFAULT_MINB_ANN) {
    case 6: return f(k_ann_clip_b<6>);
    case 8: return f(k_ann_clip_b<8>);
    default: return f(k_ann_clip);
    }
}

cudaError_t launch_ann_clip(const AnnClipArgs& a, bool big, int grid, int block, cudaStream_t s)
{
    if (big) k_ann_clip_big<<<grid, block, 0, s>>>(a);
    else ann_variant([&](auto k) { k<<<grid, block, 0, s>>>(a); return 0; });
    return cudaGetLastError();
}

size_t ann_scratch_bytes(bool big) { return big ? ann_region_bytes<NS_BIG>() : ann_region_bytes<NS_MAIN>(); }

int ann_blocks_per_sm(bool big, int block)
{
    int n = 0;
    cudaError_t e = big ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_ann_clip_big, block, 0)
                        : ann_variant([&](auto k) { return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, block, 0); });
    if (e != cudaSuccess) { cudaGetLastError(); return 1; }
    return n > 0 ? n : 1;
}

// ---- each voxel's records summed into m in key order (m += w m0, src/geometry.c:249-251) ----

__global__ void k_ann_apply(ApplyArgs a)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < a.nruns; r += stride) {
        const unsigned v = a.run_vox[r];
        const long long b = a.run_off[r], n = a.run_cnt[r];
        double m = a.M[v];
        for (long long i = b; i < b + n; ++i) m += a.mom[i];
        a.M[v] = m;
    }
}

cudaError_t launch_ann_apply(const ApplyArgs& a, cudaStream_t s)
{
    k_ann_apply<<<grid_for(a.nruns, 128), 128, 0, s>>>(a);
    return cudaGetLastError();
}

} // namespace psib
