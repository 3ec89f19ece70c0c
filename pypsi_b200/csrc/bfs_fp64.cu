// bfs_fp64.cu -- the FP64 clip of the main tet images as a breadth-first walk
// of their bisection trees, bit for bit the depth-first FP64 kernel's
// fragments (psib_clip.cuh, after psi_voxelize_tet, src/geometry.c:60-188).
//
// The walk is the mixed one's (bfs.cu: one cut per polyhedron per level
// launch, 32-wide queue tiles, warp-wide reservation of queue elements), with
// the depth-first FP64 kernel's arithmetic: FP64 positions in the image's own
// coordinates and FP64 q for every vertex, window planes cut first and in
// the order x-low, x-high, y-low, ... as they are found, the middle grid
// plane of the longest axis after them, and every cut vertex interpolated as
// cut_poly does, in the reference's operation order (src/geometry.c:441-445,
// :601-605).  This unit is compiled without FMA contraction, as the other
// FP64 units are.  The split plane of a node depends only on its index box,
// so every fragment is cut by the same planes in the same order, and holds
// the same vertices in the same order, as in the depth-first walk; its
// moments (reduce_poly, src/geometry.c:692-767) and its record -- key (voxel,
// image), the raw moments about q = 0 -- are then those of the depth-first
// walk bit for bit, and sorting the records by key restores the reference's
// order of the field update (src/geometry.c:164-186).
//
// Queue elements hold six FP64 words per vertex (position, q), so a pass
// takes fewer images than the mixed walk's; the host sizes passes by the
// same box-volume bound.
#include "psib_bfs.cuh"
#include "psib_device.cuh"
#include "psib_kernels.h"

namespace psib {

__device__ __forceinline__ size_t qd(unsigned long long e, int v, int c)
{
    return ((size_t)(e >> 5) * (MAXV * 6) + (size_t)(v * 6 + c)) * 32 + (size_t)(e & 31);
}
// queue element bytes: positions, q and links of nv vertices, nv, window mask, box, image
__device__ __forceinline__ unsigned long long elem_bytes64(int nv) { return 52ull * nv + 18ull; }

// ---- init: tet images -> first polyhedra ----

__global__ void __launch_bounds__(BB) k_bfs64_init(BfsArgs a)
{
    const int lane = threadIdx.x & 31;
    const long long warp = (long long)blockIdx.x * (BB / 32) + (threadIdx.x >> 5);
    const long long nwarp = (long long)gridDim.x * (BB / 32);
    const unsigned long long pass = *a.pass_idx;
    const long long q0 = a.passes[pass], q1 = a.passes[pass + 1];
    unsigned st = 0;
    unsigned long long moved = 0;
    for (long long base = q0 + warp * 32; base < q1; base += nwarp * 32) {
        const long long i = base + lane;
        const bool act = i < q1;
        int t = 0;
        double p[4][3];
        int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        uint32_t wmask = 0; // window planes: bit 2a keeps x_a >= w0_a, bit 2a+1 keeps x_a <= w1_a
        if (act) {
            t = a.c.order[i];
            const GridDev& g = grid_of(a.c, t);
            const double* fr = a.c.it.frame + (size_t)t * FRAME;
            for (int v = 0; v < 4; ++v)
                for (int c = 0; c < 3; ++c) p[v][c] = fr[3 * v + c];
            // window planes and index box as the depth-first walk computes them (src/geometry.c:816-842)
            for (int c = 0; c < 3; ++c) {
                double cmin = 1.0e30, cmax = -1.0e30;
                for (int v = 0; v < 4; ++v) {
                    if (p[v][c] < cmin) cmin = p[v][c];
                    if (p[v][c] > cmax) cmax = p[v][c];
                }
                const bool clo = g.w0[c] > cmin, chi = g.w1[c] < cmax;
                wmask |= (clo ? 1u : 0u) << (2 * c) | (chi ? 1u : 0u) << (2 * c + 1);
                if (clo) cmin = g.w0[c];
                if (chi) cmax = g.w1[c];
                lo[c] = (int)floor((cmin - g.w0[c]) / g.d[c]);
                hi[c] = (int)ceil((cmax - g.w0[c]) / g.d[c]);
                if (lo[c] < 0) lo[c] = 0;
                if (hi[c] > g.n[c]) hi[c] = g.n[c];
                if (hi[c] < lo[c]) hi[c] = lo[c]; // wholly outside: the window cut finds it empty
            }
        }
        const bool leaf = act && wmask == 0 && one_voxel(lo, hi);
        unsigned oq, ol;
        const unsigned long long bq = warp_reserve(a.out.count, act && !leaf ? 1u : 0u, oq);
        const unsigned long long bl = warp_reserve(a.leaf.count, leaf ? 1u : 0u, ol);
        if (act) {
            const PolyQueue& Q = leaf ? a.leaf : a.out;
            const unsigned long long e = leaf ? bl + ol : bq + oq;
            if (e >= Q.cap) {
                st |= ST_OVERFLOW;
            } else {
                // the tet's vertex graph (src/geometry.c:776-787), q = (0, e_x, e_y, e_z), plane tags
                const uint32_t links[4] = {1u | (3u << 8) | (2u << 16), 2u | (3u << 8) | (0u << 16),
                                           0u | (3u << 8) | (1u << 16), 1u | (2u << 8) | (0u << 16)};
                for (int v = 0; v < 4; ++v) {
                    for (int c = 0; c < 3; ++c) {
                        Q.xq[qd(e, v, c)] = p[v][c];
                        Q.xq[qd(e, v, 3 + c)] = (v == c + 1) ? 1.0 : 0.0;
                    }
                    Q.nb[qn(e, v)] = links[v] | ((0xFu & ~(1u << v)) << 24);
                }
                Q.nv[e] = 4;
                moved += 96 + elem_bytes64(4);
                Q.win[e] = (uint8_t)wmask;
                put_box(Q, e, lo, hi);
                Q.item[e] = (uint32_t)t;
            }
        }
    }
    if (st) atomicOr(a.c.status, st);
    if (a.bytes && moved) atomicAdd(a.bytes, moved);
}

// ---- level: one cut per polyhedron ----

// The signed distance of vertex v of element e of Q from the current plane, as the depth-first
// walk computes it: a window plane (win >= 0: bit 2 ax + side) is
// ((d + x0 n0) + x1 n1) + x2 n2 with n = +-e_ax and d = -w0 or w1 (src/geometry.c:391-501);
// the middle grid plane is cr - x_ax.
__device__ __forceinline__ double plane_dist(const PolyQueue& Q, unsigned long long e, int v, int win, int ax,
                                             double cr)
{
    if (win < 0) return cr - Q.xq[qd(e, v, ax)];
    const double sg = (win & 1) ? -1.0 : 1.0;
    double t0 = cr;
    for (int i = 0; i < 3; ++i) t0 += Q.xq[qd(e, v, i)] * (i == ax ? sg : 0.0);
    return t0;
}

// Cut the polyhedron at element eI of the input queue (links staged in nbI; upper side = bits
// of um, distances from plane_dist) into element el of QL (lower side, s >= 0) and, when
// keep_up, eu of QU (upper side), with the vertex order and arithmetic of cut_poly.
__device__ __forceinline__ unsigned bfs64_cut(int nv, uint32_t um, int win, int ax, double cr, const PolyQueue& QI,
                                              unsigned long long eI, const uint32_t* nbI, uint32_t* nbL,
                                              uint32_t* nbU, const PolyQueue& QL, unsigned long long el,
                                              const PolyQueue& QU, unsigned long long eu, bool keep_up,
                                              uint32_t cut_tag, uint64_t cm, int& cntL, int& cntU)
{
    const uint32_t lmask = ((1u << nv) - 1u) & ~um;
    const int nl = __popc(lmask), nu = __popc(um);
    // a failure ends the loops through err rather than a return (the lanes of a warp then leave
    // every loop at one place)
    unsigned err = 0;
    for (int v = 0; v < nv && !err; ++v) {
        const bool u = (um >> v) & 1u;
        const uint32_t sm = u ? um : lmask;
        const int j = rank_in(sm, v);
        const PolyQueue& Q = u ? QU : QL;
        const unsigned long long d = u ? eu : el;
        if (!u || keep_up)
            for (int c = 0; c < 6; ++c) Q.xq[qd(d, j, c)] = QI.xq[qd(eI, v, c)];
        const uint32_t w = AT(nbI, v);
        uint32_t ow = 0xFFFFFFu | (w & ALL_TAGS);
        for (int k = 0; k < 3; ++k) {
            const int t = nbget(w, k);
            if (t >= nv) {
                err = ST_GRAPH;
                break;
            }
            if ((((um >> t) & 1u) != 0) == u) ow = nbset(ow, k, rank_in(sm, t));
        }
        if (u) AT(nbU, j) = ow;
        else AT(nbL, j) = ow;
    }
    // the cut edges lowest bit first: cut_poly's order of the new vertices
    int k = 0;
    while (cm && !err) {
        const int bit = __ffsll((long long)cm) - 1;
        cm &= cm - 1ull;
        const int vc = bit / 3, np = bit - 3 * vc;
        const uint32_t w = AT(nbI, vc);
        const int jc = rank_in(lmask, vc);
        const int vn = nbget(w, np);
        if (nl + k >= MAXV || nu + k >= MAXV) {
            err = ST_OVERFLOW;
            break;
        }
        const double sc = plane_dist(QI, eI, vc, win, ax, cr), sn = plane_dist(QI, eI, vn, win, ax, cr);
        const double iw = 1.0 / (sc - sn);
        for (int c = 0; c < 6; ++c) {
            const double px = iw * (QI.xq[qd(eI, vn, c)] * sc - QI.xq[qd(eI, vc, c)] * sn);
            QL.xq[qd(el, nl + k, c)] = px;
            if (keep_up) QU.xq[qd(eu, nu + k, c)] = px;
        }
        const uint32_t wn = AT(nbI, vn);
        const uint32_t tg = (w & wn & ALL_TAGS) | cut_tag;
        AT(nbL, nl + k) = 0xFFFF00u | (uint32_t)jc | tg;
        AT(nbL, jc) = nbset(AT(nbL, jc), np, nl + k);
        const int jn = rank_in(um, vn);
        AT(nbU, nu + k) = 0xFFFF00u | (uint32_t)jn | tg;
        const int kb = (nbget(wn, 0) == vc) ? 0 : (nbget(wn, 1) == vc) ? 1 : (nbget(wn, 2) == vc) ? 2 : 3;
        if (kb == 3) {
            err = ST_GRAPH;
            break;
        }
        AT(nbU, jn) = nbset(AT(nbU, jn), kb, nu + k);
        ++k;
    }
    if (!err && (!link_cut_shared(nbL, nl, nl + k) || (keep_up && !link_cut_shared(nbU, nu, nu + k))))
        err = ST_GRAPH;
    if (err) return err;
    for (int v = 0; v < nl + k; ++v) QL.nb[qn(el, v)] = AT(nbL, v);
    QL.nv[el] = (uint8_t)(nl + k);
    cntL = nl + k;
    if (keep_up) {
        for (int v = 0; v < nu + k; ++v) QU.nb[qn(eu, v)] = AT(nbU, v);
        QU.nv[eu] = (uint8_t)(nu + k);
        cntU = nu + k;
    }
    return 0;
}

__global__ void __launch_bounds__(BB) k_bfs64_level(BfsArgs a)
{
    extern __shared__ uint32_t smem[];
    uint32_t* nbI = smem;
    uint32_t* nbL = smem + MAXV * BB;
    uint32_t* nbU = smem + 2 * MAXV * BB;
    const long long warp = (long long)blockIdx.x * (BB / 32) + (threadIdx.x >> 5);
    const long long nwarp = (long long)gridDim.x * (BB / 32);
    // a producer reserves before it checks capacity (and flags the overflow), so clamp
    const unsigned long long n = min(*a.in.count, a.in.cap);
    unsigned st = 0;
    unsigned long long splits = 0, moved = 0;
    for (unsigned long long base = (unsigned long long)warp * 32; base < n; base += (unsigned long long)nwarp * 32) {
        const unsigned long long e = base + (threadIdx.x & 31);
        bool act = e < n;
        int nv = 0, lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, ax = 0, nlo = 0, nup = 0, pl = -1;
        uint32_t um = 0, t = 0, win = 0;
        double cr = 0.0;
        bool cut = false, toleaf = false, wcut = false;
        if (act) {
            nv = a.in.nv[e];
            if (nv < 4 || nv > MAXV) act = false; // a failed cut upstream (status already set)
        }
        if (act) {
            get_box(a.in, e, lo, hi);
            moved += elem_bytes64(nv);
            t = a.in.item[e];
            const GridDev& g = grid_of(a.c, t);
            for (int v = 0; v < nv; ++v) AT(nbI, v) = a.in.nb[qn(e, v)];
            win = a.in.win[e];
            const uint32_t all = (1u << nv) - 1u;
            for (int guard = 0; guard < 64; ++guard) {
                if (win) {
                    // a pending window plane: skipped when no vertex is below it, the image is
                    // empty when none is above it, as in the depth-first window clip
                    pl = __ffs(win) - 1;
                    win &= ~(1u << pl);
                    ax = pl >> 1;
                    cr = (pl & 1) ? g.w1[ax] : -g.w0[ax];
                    um = 0;
                    uint32_t zm = 0;
                    for (int v = 0; v < nv; ++v) {
                        const double s = plane_dist(a.in, e, v, pl, ax, cr);
                        if (s < 0.0) um |= 1u << v;
                        if (s <= 0.0) zm |= 1u << v;
                    }
                    if (um == 0) continue;
                    if (zm == all) { act = false; break; }
                    wcut = true;
                    break;
                }
                pl = -1;
                int dmax = 0;
                ax = 0;
                for (int c = 0; c < 3; ++c) {
                    const int sz = hi[c] - lo[c];
                    if (sz > dmax) { dmax = sz; ax = c; }
                }
                if (dmax <= 1) { toleaf = true; break; }
                ++splits;
                // the middle grid plane of the longest axis (src/geometry.c:886-893)
                cr = g.d[ax] * (lo[ax] + dmax / 2) + g.w0[ax];
                um = 0;
                for (int v = 0; v < nv; ++v)
                    if (cr - a.in.xq[qd(e, v, ax)] < 0.0) um |= 1u << v;
                nlo = dmax / 2;
                nup = dmax - nlo;
                if (um == 0) { hi[ax] -= nup; continue; }
                if (um == all) { lo[ax] += nlo; continue; }
                cut = true;
                break;
            }
            if (act && !cut && !toleaf && !wcut) { st |= ST_DEPTH; act = false; }
        }
        if (!act) { cut = toleaf = wcut = false; }
        int llo[3], lhi[3], ulo[3], uhi[3];
        for (int c = 0; c < 3; ++c) { llo[c] = ulo[c] = lo[c]; lhi[c] = uhi[c] = hi[c]; }
        if (cut) { lhi[ax] -= nup; ulo[ax] += nlo; }
        const bool leafL = (cut && one_voxel(llo, lhi)) || (wcut && !win && one_voxel(lo, hi));
        const bool leafU = cut && one_voxel(ulo, uhi);
        const bool lfL = toleaf || leafL, lfU = cut && leafU; // toleaf: the polyhedron itself, as "L"
        const bool qL = (cut || wcut) && !leafL, qU = cut && !leafU;
        const unsigned nq = (unsigned)qL + (unsigned)qU;
        const unsigned nlf = (unsigned)lfL + (unsigned)lfU;
        if (a.last && nq) st |= ST_DEPTH;
        unsigned oq, ol;
        const unsigned long long bq = warp_reserve(a.out.count, nq, oq);
        const unsigned long long bl = warp_reserve(a.leaf.count, nlf, ol);
        unsigned long long nextq = bq + oq, nextl = bl + ol;
        if (toleaf) {
            const unsigned long long d = nextl++;
            if (d >= a.leaf.cap) {
                st |= ST_OVERFLOW;
            } else {
                for (int v = 0; v < nv; ++v) {
                    for (int c = 0; c < 6; ++c) a.leaf.xq[qd(d, v, c)] = a.in.xq[qd(e, v, c)];
                    a.leaf.nb[qn(d, v)] = AT(nbI, v);
                }
                a.leaf.nv[d] = (uint8_t)nv;
                moved += elem_bytes64(nv);
                put_box(a.leaf, d, lo, hi);
                a.leaf.item[d] = t;
            }
        }
        if (cut || wcut) {
            // a middle-plane cut keeps both children, a window cut only the side with s >= 0
            const PolyQueue& QL = leafL ? a.leaf : a.out;
            const unsigned long long el = leafL ? nextl++ : nextq++;
            const PolyQueue& QU = !cut ? QL : leafU ? a.leaf : a.out;
            const unsigned long long eu = !cut ? el : leafU ? nextl++ : nextq++;
            if (el >= QL.cap || eu >= QU.cap) {
                st |= ST_OVERFLOW;
            } else {
                const uint64_t cm = cut_edges(nv, um, nbI);
                int nL = 0, nU = 0;
                const unsigned e2 = bfs64_cut(nv, um, cut ? -1 : pl, ax, cr, a.in, e, nbI, nbL, nbU, QL, el, QU, eu,
                                              cut, axis_tag(ax), cm, nL, nU);
                if (e2) {
                    st |= e2;
                    QL.nv[el] = 0; // downstream kernels skip these
                    if (cut) QU.nv[eu] = 0;
                } else {
                    moved += elem_bytes64(nL) + (cut ? elem_bytes64(nU) : 0ull);
                }
                put_box(QL, el, cut ? llo : lo, cut ? lhi : hi);
                QL.item[el] = t;
                QL.win[el] = cut ? (uint8_t)0 : (uint8_t)win;
                if (cut) {
                    put_box(QU, eu, ulo, uhi);
                    QU.item[eu] = t;
                    QU.win[eu] = 0;
                }
            }
        }
    }
    if (st) atomicOr(a.c.status, st);
    if (a.c.counters && splits) atomicAdd(&a.c.counters[2], splits);
    if (a.bytes && moved) atomicAdd(a.bytes, moved);
}

// ---- leaf: fragment moments and records ----

// A fragment as reduce_poly reads it: its links and q in registers and local memory.
struct LeafPoly64 {
    using real = double;
    static constexpr int CAP = MAXV;
    static constexpr bool has_q = true;
    int nv;
    uint32_t nb[MAXV];
    double q[MAXV][3];
};

__global__ void __launch_bounds__(BB) k_bfs64_leaf(BfsArgs a)
{
    const ClipArgs& c = a.c;
    const long long warp = (long long)blockIdx.x * (BB / 32) + (threadIdx.x >> 5);
    const long long nwarp = (long long)gridDim.x * (BB / 32);
    const unsigned long long n = min(*a.leaf.count, a.leaf.cap);
    unsigned st = 0;
    unsigned long long frags = 0, verts = 0, moved = 0;
    for (unsigned long long base = (unsigned long long)warp * 32; base < n; base += (unsigned long long)nwarp * 32) {
        const unsigned long long e = base + (threadIdx.x & 31);
        int nv = 0;
        if (e < n) nv = a.leaf.nv[e];
        const bool ok = e < n && nv >= 4 && nv <= MAXV;
        bool has = false;
        unsigned long long key = 0;
        double mom[10];
        if (ok) {
            int lo[3], hi[3];
            get_box(a.leaf, e, lo, hi);
            const uint32_t t = a.leaf.item[e];
            const GridDev& g = grid_of(c, t);
            LeafPoly64 P;
            P.nv = nv;
            for (int v = 0; v < nv; ++v) {
                P.nb[v] = a.leaf.nb[qn(e, v)];
                for (int i = 0; i < 3; ++i) P.q[v][i] = a.leaf.xq[qd(e, v, 3 + i)];
            }
            moved += elem_bytes64(nv);
            // a single voxel (src/geometry.c:873-884)
            const unsigned e2 = reduce_poly(P, mom, c.mom_order);
            st |= e2;
            if (!e2 && mom[0] > 0.0) {
                if (lo[0] >= g.n[0] || lo[1] >= g.n[1] || lo[2] >= g.n[2]) {
                    st |= ST_INDEX;
                } else {
                    const long long gi = (long long)(c.voff ? c.voff[c.it.grid[t]] : 0ull) +
                                         ((long long)g.n[1] * lo[0] + lo[1]) * g.n[2] + lo[2];
                    key = ((unsigned long long)gi << c.rec_ibits) | (unsigned long long)(t - c.rec_item_base);
                    has = true;
                    ++frags;
                    verts += nv;
                }
            }
        }
        unsigned off;
        const unsigned long long r0 = warp_reserve(c.rec_n, has ? 1u : 0u, off);
        if (has) {
            const unsigned long long r = r0 + off;
            if (r < c.rec_cap) {
                moved += 8ull * (1 + c.rec_nmom);
                c.rec_key[r] = key;
                double* dst = c.rec_mom + r * c.rec_nmom;
#pragma unroll
                for (int k = 0; k < 10; ++k)
                    if (k < c.rec_nmom) dst[k] = mom[k];
            } else {
                st |= ST_RECORDS;
            }
        }
    }
    if (st) atomicOr(c.status, st);
    if (c.counters && frags) {
        atomicAdd(&c.counters[0], frags);
        atomicAdd(&c.counters[1], verts);
    }
    if (a.bytes && moved) atomicAdd(a.bytes, moved);
}

// ---- launchers ----

static constexpr size_t LEVEL64_SMEM = 3 * MAXV * BB * sizeof(uint32_t); // links of the cut polyhedron and its children

// resident blocks per SM of each kernel (one full wave of grid-stride blocks)
static int g_blocks64[3] = {0, 0, 0};
static void occupancy64()
{
    if (g_blocks64[0]) return;
    cudaFuncSetAttribute(k_bfs64_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LEVEL64_SMEM);
    int b[3] = {1, 1, 1};
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b[0], k_bfs64_init, BB, 0) != cudaSuccess) b[0] = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b[1], k_bfs64_level, BB, LEVEL64_SMEM) != cudaSuccess) b[1] = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b[2], k_bfs64_leaf, BB, 0) != cudaSuccess) b[2] = 1;
    cudaGetLastError();
    for (int i = 0; i < 3; ++i) g_blocks64[i] = b[i] > 0 ? b[i] : 1;
}
void bfs64_prepare() { occupancy64(); }

cudaError_t launch_bfs64_init(const BfsArgs& a, int num_sms, cudaStream_t s)
{
    occupancy64();
    k_bfs64_init<<<num_sms * g_blocks64[0], BB, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_bfs64_level(const BfsArgs& a, int num_sms, cudaStream_t s)
{
    occupancy64();
    k_bfs64_level<<<num_sms * g_blocks64[1], BB, LEVEL64_SMEM, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_bfs64_leaf(const BfsArgs& a, int num_sms, cudaStream_t s)
{
    occupancy64();
    k_bfs64_leaf<<<num_sms * g_blocks64[2], BB, 0, s>>>(a);
    return cudaGetLastError();
}

} // namespace psib
