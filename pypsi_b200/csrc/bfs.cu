// bfs.cu -- the mixed-precision clip of the main tet images as a breadth-first
// walk of their bisection trees.
//
// The depth-first walk of one tet per thread (psib_clip.cuh) leaves most lanes
// of a warp idle, because every lane walks a tree of its own shape, and its
// per-thread stack of polyhedra does not fit in the caches.  Here each level
// of the trees is one launch in which every thread makes exactly one cut of
// one polyhedron:
//
//   init   tet image -> its first polyhedron (4 vertices, FP32 positions
//          relative to the image's vertex 0), to the level queue, or to the
//          leaf queue when its index box is one voxel; images that need the
//          window clip go to a list for the depth-first kernel
//   level  polyhedron -> shrink its box while the middle plane misses it, then
//          one cut into two children; each child goes to the next level queue
//          or, when its box is one voxel, to the leaf queue
//   leaf   fragment -> FP64 vertices from their planes, central moments, a
//          record (key voxel|image), as the depth-first mixed kernel does
//
// The split plane of a node depends only on its index box, so every fragment
// sees the same cuts in the same order as in the depth-first walk; only the
// order in which fragments are produced differs, and records are sorted by
// (voxel, image) afterwards.
//
// Queues hold polyhedra in 32-wide tiles: element e's vertex v, coordinate c
// sits at ((e/32 * MAXV + v) * 3 + c) * 32 + e%32, so the lanes of a warp,
// which hold consecutive elements, touch consecutive words.  A warp reserves
// its outputs with one atomic per queue after a warp-wide prefix sum, and
// writes them to consecutive elements.  The links of the polyhedron being cut
// and of its two children, and the positions of the one being cut, live in
// shared memory as [vertex][thread] (no bank conflicts whatever vertex each
// lane touches); the leaf kernel keeps its fragment's FP64 q there.
//
// A level queue never holds more polyhedra than the leaves its images will
// produce, which is at most the sum of their index-box volumes; the host sizes
// each pass of images by that bound.
#include "psib_accum.cuh"
#include "psib_bfs.cuh"
#include "psib_device.cuh"
#include "psib_kernels.h"

namespace psib {

// ---- init: tet images -> first polyhedra ----

// q-volume (fraction of the tet) inside the window planes of wmask, clipped in
// FP64 as the depth-first kernel's window clip does.
__device__ double window_volume(const double (*p)[3], uint32_t wmask, const GridDev& g)
{
    Poly<double> W[2];
    init_tet(W[0], p);
    int cw = 0;
    double sd[MAXV];
    for (int pl = 0; pl < 6 && W[cw].nv > 0; ++pl) {
        if (!((wmask >> pl) & 1u)) continue;
        const int ax = pl >> 1;
        const bool lo_side = !(pl & 1);
        double smin = 1.0e30, smax = -1.0e30;
        uint32_t um = 0;
        for (int v = 0; v < W[cw].nv; ++v) {
            const double t0 = lo_side ? W[cw].x[v][ax] - g.w0[ax] : g.w1[ax] - W[cw].x[v][ax];
            sd[v] = t0;
            if (t0 < smin) smin = t0;
            if (t0 > smax) smax = t0;
            if (t0 < 0.0) um |= 1u << v;
        }
        if (smin >= 0.0) continue;
        if (smax <= 0.0) return 0.0;
        if (cut_poly<double, false>(W[cw], sd, um, W[1 - cw], W[1 - cw], axis_tag(ax))) return 0.0;
        cw = 1 - cw;
    }
    double m[10];
    if (reduce_poly(W[cw], m, 0)) return 0.0;
    return m[0];
}

__global__ void __launch_bounds__(BB) k_bfs_init(BfsArgs a)
{
    const int lane = threadIdx.x & 31;
    const long long warp = (long long)blockIdx.x * (BB / 32) + (threadIdx.x >> 5);
    const long long nwarp = (long long)gridDim.x * (BB / 32);
    const unsigned long long p = *a.pass_idx;
    const long long q0 = a.passes[p], q1 = a.passes[p + 1];
    unsigned st = 0;
    unsigned long long moved = 0;
    for (long long base = q0 + warp * 32; base < q1; base += nwarp * 32) {
        const long long i = base + lane;
        const bool act = i < q1;
        int t = 0;
        double p[4][3];
        int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        bool window = false;
        const GridDev* gp = &a.c.g;
        uint32_t wmask = 0; // window planes: bit 2a keeps x_a >= w0_a, bit 2a+1 keeps x_a <= w1_a
        if (act) {
            t = a.c.order[i];
            gp = &grid_of(a.c, t);
            const double* fr = a.c.it.frame + (size_t)t * FRAME;
            for (int v = 0; v < 4; ++v)
                for (int c = 0; c < 3; ++c) p[v][c] = fr[3 * v + c];
            // window planes and index box as the depth-first walk computes them (src/geometry.c:816-842)
            for (int c = 0; c < 3; ++c) {
                double cmin = p[0][c], cmax = p[0][c];
                for (int v = 1; v < 4; ++v) {
                    if (p[v][c] < cmin) cmin = p[v][c];
                    if (p[v][c] > cmax) cmax = p[v][c];
                }
                const bool clo = gp->w0[c] > cmin, chi = gp->w1[c] < cmax;
                window = window || clo || chi;
                wmask |= (clo ? 1u : 0u) << (2 * c) | (chi ? 1u : 0u) << (2 * c + 1);
                if (clo) cmin = gp->w0[c];
                if (chi) cmax = gp->w1[c];
                lo[c] = (int)floor((cmin - gp->w0[c]) / gp->d[c]);
                hi[c] = (int)ceil((cmax - gp->w0[c]) / gp->d[c]);
                if (lo[c] < 0) lo[c] = 0;
                if (hi[c] > gp->n[c]) hi[c] = gp->n[c];
                if (hi[c] < lo[c]) hi[c] = lo[c];
            }
        }
        // the exact FP64 q-volume of a window-clipped image: its mass correction target
        double target = 1.0;
        const bool wbfs = act && window && a.window_bfs;
        if (wbfs) target = window_volume(p, wmask, *gp);
        const bool to_dfs = act && window && !a.window_bfs;
        const bool use = act && (!window || (wbfs && target > 0.0));
        const bool leaf = use && !wbfs && one_voxel(lo, hi);
        unsigned od, oq, ol;
        const unsigned long long bd = warp_reserve(a.dfs_count, to_dfs ? 1u : 0u, od);
        const unsigned long long bq = warp_reserve(a.out.count, use && !leaf ? 1u : 0u, oq);
        const unsigned long long bl = warp_reserve(a.leaf.count, leaf ? 1u : 0u, ol);
        if (to_dfs) a.dfs_list[bd + od] = t;
        // the correction pass walks images again with their mass factor: their scale stays as it is
        const bool main_pass = a.c.acc.factor == nullptr;
        if (wbfs && !use && main_pass) a.c.scale[t] = 1.0; // wholly outside the window: deposits nothing
        if (use) {
            if (main_pass) {
                a.c.scale[t] = -target; // marks a breadth-first image: bfs_finalize sets its mass correction
                a.vsum[t] = 0.0;
            }
            const PolyQueue& Q = leaf ? a.leaf : a.out;
            const unsigned long long e = leaf ? bl + ol : bq + oq;
            if (e >= Q.cap) {
                st |= ST_OVERFLOW;
            } else {
                // the tet's vertex graph (src/geometry.c:776-787) with its plane tags
                const uint32_t links[4] = {1u | (3u << 8) | (2u << 16), 2u | (3u << 8) | (0u << 16),
                                           0u | (3u << 8) | (1u << 16), 1u | (2u << 8) | (0u << 16)};
                for (int v = 0; v < 4; ++v) {
                    for (int c = 0; c < 3; ++c) Q.x[qx(e, v, c)] = (float)(p[v][c] - p[0][c]);
                    Q.nb[qn(e, v)] = links[v] | ((0xFu & ~(1u << v)) << 24);
                }
                Q.nv[e] = 4;
                moved += 96 + elem_bytes(4);
                Q.win[e] = (uint8_t)(wbfs ? wmask : 0u);
                put_box(Q, e, lo, hi);
                Q.item[e] = (uint32_t)t;
            }
        }
    }
    if (st) atomicOr(a.c.status, st);
    if (a.bytes && moved) atomicAdd(a.bytes, moved);
}

// ---- level: one cut per polyhedron ----

// Cut the polyhedron at element eI of the input queue (positions read from
// there, links staged in nbI; upper side = bits of um, s = cr - x[ax]) into
// element el of QL (lower side) and eu of QU (upper side), with the vertex
// order and arithmetic of cut_poly.
__device__ __forceinline__ unsigned bfs_cut(int nv, uint32_t um, float cr, float sg, int ax, const PolyQueue& QI,
                                            unsigned long long eI, const uint32_t* nbI, uint32_t* nbL, uint32_t* nbU,
                                            const PolyQueue& QL, unsigned long long el, const PolyQueue& QU,
                                            unsigned long long eu, bool keep_up, uint32_t cut_tag, uint64_t cm,
                                            int& cntL, int& cntU)
{
    auto X = [&](int v, int c) { return __ldg(&QI.x[qx(eI, v, c)]); };
    const uint32_t lmask = ((1u << nv) - 1u) & ~um;
    const int nl = __popc(lmask), nu = __popc(um);
    // a failure ends the loops through err rather than a return, so that the lanes of a warp
    // leave every loop at one place and run the next step together
    unsigned err = 0;
    for (int v = 0; v < nv && !err; ++v) {
        const bool u = (um >> v) & 1u;
        const uint32_t sm = u ? um : lmask;
        const int j = rank_in(sm, v);
        const PolyQueue& Q = u ? QU : QL;
        const unsigned long long d = u ? eu : el;
        if (!u || keep_up)
            for (int c = 0; c < 3; ++c) Q.x[qx(d, j, c)] = X(v, c);
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
    // cm: the cut edges (cut_edges); taking the lowest bit first creates the cut vertices in
    // cut_poly's order
    int k = 0;
    while (cm && !err) {
        const int bit = __ffsll((long long)cm) - 1;
        cm &= cm - 1ull;
        const int vc = bit / 3, np = bit - 3 * vc;
        const uint32_t w = AT(nbI, vc);
        const int jc = rank_in(lmask, vc);
        {
            const int vn = nbget(w, np);
            if (nl + k >= MAXV || nu + k >= MAXV) {
                err = ST_OVERFLOW;
                break;
            }
            const float sc = sg * (cr - X(vc, ax)), sn = sg * (cr - X(vn, ax));
            const float iw = 1.0f / (sc - sn);
            for (int c = 0; c < 3; ++c) {
                const float px = iw * (X(vn, c) * sc - X(vc, c) * sn);
                QL.x[qx(el, nl + k, c)] = px;
                if (keep_up) QU.x[qx(eu, nu + k, c)] = px;
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

__global__ void __launch_bounds__(BB, 7) k_bfs_level(BfsArgs a)
{
    extern __shared__ uint32_t smem[];
    uint32_t* nbI = smem;
    uint32_t* nbL = smem + MAXV * BB;
    uint32_t* nbU = smem + 2 * MAXV * BB;
    const int lane = threadIdx.x & 31;
    const long long warp = (long long)blockIdx.x * (BB / 32) + (threadIdx.x >> 5);
    const long long nwarp = (long long)gridDim.x * (BB / 32);
    // a producer reserves before it checks capacity (and flags the overflow), so clamp; the input
    // queue's two ends: [0, ilo) and, for polyhedra of more vertices, its last ihi elements
    const unsigned long long ilo = min(*a.in.count, a.in.cap);
    unsigned long long ihi = a.in.count_hi ? min(*a.in.count_hi, a.in.cap) : 0ull;
    unsigned st = 0;
    if (ilo + ihi > a.in.cap) { // the ends met: more polyhedra than a pass can hold
        st |= ST_OVERFLOW;
        ihi = a.in.cap - ilo;
    }
    const unsigned long long n = ilo + ihi;
    unsigned long long splits = 0, moved = 0;
    for (unsigned long long base = (unsigned long long)warp * 32; base < n; base += (unsigned long long)nwarp * 32) {
        const unsigned long long ie = base + lane;
        const unsigned long long e = ie < ilo ? ie : a.in.cap - 1ull - (ie - ilo);
        bool act = ie < n;
        int nv = 0, lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, ax = 0, nlo = 0, nup = 0;
        uint32_t um = 0, t = 0, win = 0;
        float cr = 0.0f, sg = 1.0f;
        bool cut = false, toleaf = false, wcut = false;
        if (act) {
            nv = a.in.nv[e];
            if (nv < 4 || nv > MAXV) act = false; // a failed cut upstream (status already set)
        }
        if (act) {
            get_box(a.in, e, lo, hi);
            moved += elem_bytes(nv);
            t = a.in.item[e];
            const GridDev& g = grid_of(a.c, t);
            const double* fr = a.c.it.frame + (size_t)t * FRAME; // vertex 0: the origin of the FP32 positions
            // the links are staged (the cut walks them); positions are read from the queue
            for (int v = 0; v < nv; ++v) AT(nbI, v) = a.in.nb[qn(e, v)];
            win = a.in.win[e];
            for (int guard = 0; guard < 64; ++guard) {
                if (win) {
                    // a pending window plane, kept side s >= 0 as in the window clip
                    // (src/geometry.c:391-501): s = x - w0 or w1 - x
                    const int pl = __ffs(win) - 1;
                    win &= ~(1u << pl);
                    ax = pl >> 1;
                    const bool lo_side = !(pl & 1);
                    cr = (float)((lo_side ? g.w0[ax] : g.w1[ax]) - fr[ax]);
                    sg = lo_side ? -1.0f : 1.0f;
                    um = 0;
                    for (int v = 0; v < nv; ++v)
                        if (sg * (cr - __ldg(&a.in.x[qx(e, v, ax)])) < 0.0f) um |= 1u << v;
                    if (um == 0) continue;                   // wholly inside this plane
                    if (um == (1u << nv) - 1u) { act = false; break; } // wholly outside
                    wcut = true;
                    break;
                }
                sg = 1.0f;
                int dmax = 0;
                ax = 0;
                for (int c = 0; c < 3; ++c) {
                    const int sz = hi[c] - lo[c];
                    if (sz > dmax) { dmax = sz; ax = c; }
                }
                if (dmax <= 1) { toleaf = true; break; }
                ++splits;
                // the middle grid plane of the longest axis (src/geometry.c:886-893)
                const double coord = g.d[ax] * (lo[ax] + dmax / 2) + g.w0[ax];
                cr = (float)(coord - fr[ax]);
                um = 0;
                for (int v = 0; v < nv; ++v)
                    if (cr - __ldg(&a.in.x[qx(e, v, ax)]) < 0.0f) um |= 1u << v;
                nlo = dmax / 2;
                nup = dmax - nlo;
                if (um == 0) { hi[ax] -= nup; continue; }
                if (um == (1u << nv) - 1u) { lo[ax] += nlo; continue; }
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
        // the children's vertex counts, known before the cut: each side's vertices plus one per cut edge
        uint64_t cm = 0ull;
        int nvL = nv, nvU = 0;
        if (cut || wcut) {
            cm = cut_edges(nv, um, nbI);
            const int kc = __popcll((long long)cm);
            nvL = __popc(((1u << nv) - 1u) & ~um) + kc;
            nvU = __popc(um) + kc;
        }
        // leaf children go to the low end (few vertices) or the high end of the leaf queue
        const bool hiL = a.leaf_split > 0 && nvL > a.leaf_split, hiU = a.leaf_split > 0 && nvU > a.leaf_split;
        const bool lfL = toleaf || leafL, lfU = cut && leafU; // toleaf: the polyhedron itself, as "L"
        // the next level queue is filled from both ends the same way
        const bool qL = (cut || wcut) && !leafL, qU = cut && !leafU;
        const bool two = a.out.count_hi != nullptr && a.level_split > 0; // the level queue's high end
        const bool qhL = two && nvL > a.level_split, qhU = two && nvU > a.level_split;
        const unsigned nq = (unsigned)qL + (unsigned)qU;
        const unsigned nq_lo = (unsigned)(qL && !qhL) + (unsigned)(qU && !qhU);
        const unsigned nq_hi = nq - nq_lo;
        const unsigned nleaf_lo = (unsigned)(lfL && !hiL) + (unsigned)(lfU && !hiU);
        const unsigned nleaf_hi = (unsigned)(lfL && hiL) + (unsigned)(lfU && hiU);
        if (a.last && nq) st |= ST_DEPTH;
        unsigned oq, oqh, ol, oh;
        const unsigned long long bq = warp_reserve(a.out.count, nq_lo, oq);
        const unsigned long long bqh = two ? warp_reserve(a.out.count_hi, nq_hi, oqh) : 0ull;
        if (!two) oqh = 0;
        const unsigned long long bl = warp_reserve(a.leaf.count, nleaf_lo, ol);
        const unsigned long long bh = warp_reserve(a.leaf.count_hi, nleaf_hi, oh);
        // element of the next child of this lane at the low or high end of queue Q (false: past it)
        unsigned li = 0, hj = 0, qi = 0, qj = 0;
        auto end_slot = [](const PolyQueue& Q, bool high, unsigned long long b_lo, unsigned o_lo, unsigned& i_lo,
                           unsigned long long b_hi, unsigned o_hi, unsigned& i_hi, unsigned long long& d) -> bool {
            if (!high) {
                d = b_lo + o_lo + i_lo++;
                return d < Q.cap;
            }
            const unsigned long long j = b_hi + o_hi + i_hi++;
            d = Q.cap - 1ull - j;
            return j < Q.cap;
        };
        auto leaf_slot = [&](bool high, unsigned long long& d) -> bool {
            return end_slot(a.leaf, high, bl, ol, li, bh, oh, hj, d);
        };
        auto out_slot = [&](bool high, unsigned long long& d) -> bool {
            return end_slot(a.out, high, bq, oq, qi, bqh, oqh, qj, d);
        };
        if (toleaf) {
            unsigned long long d = 0;
            if (!leaf_slot(hiL, d)) {
                st |= ST_OVERFLOW;
            } else {
                for (int v = 0; v < nv; ++v) {
                    for (int c = 0; c < 3; ++c) a.leaf.x[qx(d, v, c)] = __ldg(&a.in.x[qx(e, v, c)]);
                    a.leaf.nb[qn(d, v)] = AT(nbI, v);
                }
                a.leaf.nv[d] = (uint8_t)nv;
                moved += elem_bytes(nv);
                put_box(a.leaf, d, lo, hi);
                a.leaf.item[d] = t;
            }
        }
        if (cut || wcut) {
            // a middle-plane cut keeps both children, a window cut only the side with s >= 0; one
            // call site for both, so that lanes doing either run the cut together
            bool fits = true;
            const PolyQueue& QL = leafL ? a.leaf : a.out;
            unsigned long long el = 0;
            if (leafL) fits = leaf_slot(hiL, el);
            else fits = out_slot(qhL, el);
            const PolyQueue& QU = !cut ? QL : leafU ? a.leaf : a.out;
            unsigned long long eu = el;
            if (cut) {
                if (leafU) fits = leaf_slot(hiU, eu) && fits;
                else fits = out_slot(qhU, eu) && fits;
            }
            if (!fits) {
                st |= ST_OVERFLOW;
            } else {
                int nL = 0, nU = 0;
                const unsigned e2 = bfs_cut(nv, um, cr, cut ? 1.0f : sg, ax, a.in, e, nbI, nbL, nbU, QL, el, QU, eu,
                                            cut, axis_tag(ax), cm, nL, nU);
                if (e2) {
                    st |= e2;
                    QL.nv[el] = 0; // downstream kernels skip these
                    if (cut) QU.nv[eu] = 0;
                } else {
                    moved += elem_bytes(nL) + (cut ? elem_bytes(nU) : 0ull);
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

struct D3 {
    double x, y, z;
};

// The FP64 q of a leaf vertex beyond the shared-memory cache from its FP32
// position x (relative to the image's vertex 0) and tags w; fr is the image's
// frame, (d, w0) its grid's cell and origin, lo the fragment's voxel.  Out of
// line and with plain scalar arguments, so that the rare call neither raises
// the register count of the loop that makes it nor copies the kernel's
// arguments to local memory.
__device__ __noinline__ D3 leaf_q_slow(const double* fr, float x0, float x1, float x2, uint32_t w, double d0,
                                       double d1, double d2, double o0, double o1, double o2, int l0, int l1, int l2)
{
    const double d[3] = {d0, d1, d2}, w0[3] = {o0, o1, o2};
    const int lo[3] = {l0, l1, l2};
    double p0[3], DX[3][3], plo[3], phi[3], tol[3];
    for (int i = 0; i < 3; ++i) p0[i] = fr[i];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) DX[i][j] = fr[3 * (j + 1) + i] - p0[i];
    for (int i = 0; i < 3; ++i) {
        plo[i] = d[i] * lo[i] + w0[i];
        phi[i] = d[i] * (lo[i] + 1) + w0[i];
        tol[i] = 1.0e-3 * d[i];
    }
    const float x[3] = {x0, x1, x2};
    double q[3];
    exact_q(x, w, p0, DX, p0, plo, phi, tol, q);
    return D3{q[0], q[1], q[2]};
}

// Moments (order 0..2) of the fragment about q-point o (the q of vertex 0),
// by the fan triangles of reduce_about; the vertices' FP64 q are in qs as
// [v * 3 + c][thread] for v < QC, and solved again where a walk meets a
// vertex beyond the cache (leaf_q_slow).
template <int QC>
__device__ __forceinline__ unsigned leaf_moments(int nv, const uint32_t* nbs, const double* qs, int order, double* o,
                                                 double* mom, const BfsArgs& a, unsigned long long e, uint32_t t,
                                                 const int* lo)
{
    auto Q = [&](int v) -> D3 {
        if (QC >= MAXV || v < QC) return D3{AT(qs, 3 * v), AT(qs, 3 * v + 1), AT(qs, 3 * v + 2)};
        const GridDev& g = grid_of(a.c, t);
        return leaf_q_slow(a.c.it.frame + (size_t)t * FRAME, a.leaf.x[qx(e, v, 0)], a.leaf.x[qx(e, v, 1)],
                           a.leaf.x[qx(e, v, 2)], AT(nbs, v), g.d[0], g.d[1], g.d[2], g.w0[0], g.w0[1], g.w0[2],
                           lo[0], lo[1], lo[2]);
    };
    for (int i = 0; i < 3; ++i) o[i] = AT(qs, i);
    for (int i = 0; i < 10; ++i) mom[i] = 0.0;
    // directed edges not yet walked (3 * MAXV = 60 bits); the lowest first is
    // the face order of reduce_about
    uint64_t todo = (3 * nv >= 64) ? ~0ull : ((1ull << (3 * nv)) - 1ull);
    // a broken graph ends the loops through err rather than a return (the lanes of a warp then
    // leave each loop at one place)
    unsigned err = 0;
    while (todo && !err) {
        const int b0 = __ffsll((long long)todo) - 1;
        todo &= todo - 1ull;
        const int vs = b0 / 3, ks = b0 - 3 * vs;
        int vc = vs;
        int vn = nbget(AT(nbs, vc), ks);
        if (vn >= nv) {
            err = ST_GRAPH;
            break;
        }
        const D3 Q0 = Q(vs);
        const double q0x = Q0.x - o[0], q0y = Q0.y - o[1], q0z = Q0.z - o[2];
        uint32_t w = AT(nbs, vn);
        int k = (nbget(w, 0) == vc) ? 0 : (nbget(w, 1) == vc) ? 1 : (nbget(w, 2) == vc) ? 2 : 3;
        if (k == 3) {
            err = ST_GRAPH;
            break;
        }
        vc = vn;
        int kn = k == 2 ? 0 : k + 1;
        todo &= ~(1ull << (3 * vc + kn));
        vn = nbget(AT(nbs, vc), kn);
        int steps = 0;
        while (vn != vs) {
            if (++steps > WALK_CAP || vn >= nv) {
                err = ST_GRAPH;
                break;
            }
            const D3 Q1 = Q(vn), Q2 = Q(vc);
            const double q1x = Q1.x - o[0], q1y = Q1.y - o[1], q1z = Q1.z - o[2];
            const double q2x = Q2.x - o[0], q2y = Q2.y - o[1], q2z = Q2.z - o[2];
            const double m = (-q2x * q1y * q0z + q1x * q2y * q0z + q2x * q0y * q1z
                              - q0x * q2y * q1z - q1x * q0y * q2z + q0x * q1y * q2z);
            mom[0] += m;
            // the tet (o, q0, q1, q2): first moments m s / 4 and second moments
            // m (sum_i q_i q_i^T + s s^T) / 20 with s = q0 + q1 + q2 -- the terms of
            // reduce_about, grouped so that each takes four multiply-adds
            const double sx = q0x + q1x + q2x, sy = q0y + q1y + q2y, sz = q0z + q1z + q2z;
            if (order > 0) {
                const double h = 0.25 * m;
                mom[1] += h * sx;
                mom[2] += h * sy;
                mom[3] += h * sz;
            }
            if (order > 1) {
                const double h = 0.05 * m;
                mom[4] += h * (q0x * q0x + q1x * q1x + q2x * q2x + sx * sx);
                mom[5] += h * (q0x * q0y + q1x * q1y + q2x * q2y + sx * sy);
                mom[6] += h * (q0x * q0z + q1x * q1z + q2x * q2z + sx * sz);
                mom[7] += h * (q0y * q0y + q1y * q1y + q2y * q2y + sy * sy);
                mom[8] += h * (q0y * q0z + q1y * q1z + q2y * q2z + sy * sz);
                mom[9] += h * (q0z * q0z + q1z * q1z + q2z * q2z + sz * sz);
            }
            w = AT(nbs, vn);
            k = (nbget(w, 0) == vc) ? 0 : (nbget(w, 1) == vc) ? 1 : (nbget(w, 2) == vc) ? 2 : 3;
            if (k == 3) {
                err = ST_GRAPH;
                break;
            }
            vc = vn;
            kn = k == 2 ? 0 : k + 1;
            todo &= ~(1ull << (3 * vc + kn));
            vn = nbget(AT(nbs, vc), kn);
        }
    }
    return err;
}

// q-cache sizes of the two leaf kernels: every vertex where the kernel adds its fragments itself
// (168 registers, three blocks per SM), the first 14 where it writes records (128 registers, four
// blocks per SM: tet-voxel fragments have at most 16 vertices and 7.2 on average, so few walks
// reach past it)
constexpr int QC_REC = 14;

// INLINE: atomic mode, each fragment added to its voxel's sums here; else a record per fragment
// (sorted mode: sorted and applied after the walk).
template <bool INLINE>
__global__ void __launch_bounds__(BB, INLINE ? 3 : 4) k_bfs_leaf(BfsArgs a)
{
    constexpr int QC = INLINE ? MAXV : QC_REC;
    extern __shared__ uint32_t smem[];
    uint32_t* nbs = smem;
    double* qs = (double*)(smem + MAXV * BB); // [v * 3 + c][thread], v < QC
    const int lane = threadIdx.x & 31;
    const long long warp = (long long)blockIdx.x * (BB / 32) + (threadIdx.x >> 5);
    const long long nwarp = (long long)gridDim.x * (BB / 32);
    // the queue's two ends: [0, nlo) and, for polyhedra of more vertices, the last nhi elements
    const unsigned long long nlo = min(*a.leaf.count, a.leaf.cap);
    unsigned long long nhi = a.leaf.count_hi ? min(*a.leaf.count_hi, a.leaf.cap) : 0ull;
    const ClipArgs& c = a.c;
    unsigned st = 0;
    if (nlo + nhi > a.leaf.cap) { // the ends met: more leaves than a pass can hold
        st |= ST_OVERFLOW;
        nhi = a.leaf.cap - nlo;
    }
    const unsigned long long n = nlo + nhi;
    unsigned long long frags = 0, verts = 0, moved = 0;
    // The fragment's steps run as separate blocks -- load and vertex solves, moments, sums --
    // which every lane leaves at one place, so that lanes whose fragments have fewer vertices or
    // triangles do not start the next step apart from the rest of the warp (run that way, the
    // 28 atomics of a fragment took two passes per warp; measured 1.47x faster as blocks).
    for (unsigned long long base = (unsigned long long)warp * 32; base < n; base += (unsigned long long)nwarp * 32) {
        const unsigned long long i = base + lane;
        const unsigned long long e = i < nlo ? i : a.leaf.cap - 1ull - (i - nlo);
        bool has = false;
        double rec[10];
        unsigned long long key = 0;
        int nv = 0;
        if (i < n) nv = a.leaf.nv[e];
        const bool ok = i < n && nv >= 4 && nv <= MAXV;
        int lo[3] = {0, 0, 0}, hi[3];
        uint32_t t = 0;
        long long gi = -1; // the fragment's voxel, -1 when out of range
        const GridDev* gp = &c.g;
        if (ok) {
            get_box(a.leaf, e, lo, hi);
            t = a.leaf.item[e];
            gp = &grid_of(c, t);
            const GridDev& g = *gp;
            if (lo[0] < g.n[0] && lo[1] < g.n[1] && lo[2] < g.n[2])
                gi = (long long)(c.voff ? c.voff[c.it.grid[t]] : 0ull) +
                     ((long long)g.n[1] * lo[0] + lo[1]) * g.n[2] + lo[2];
            const double* fr = c.it.frame + (size_t)t * FRAME;
            double p0[3], DX[3][3], plo[3], phi[3], tol[3];
            for (int i = 0; i < 3; ++i) p0[i] = fr[i];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) DX[i][j] = fr[3 * (j + 1) + i] - p0[i];
            for (int i = 0; i < 3; ++i) {
                plo[i] = g.d[i] * lo[i] + g.w0[i];
                phi[i] = g.d[i] * (lo[i] + 1) + g.w0[i];
                tol[i] = 1.0e-3 * g.d[i];
            }
            for (int v = 0; v < nv; ++v) {
                const uint32_t w = a.leaf.nb[qn(e, v)];
                AT(nbs, v) = w;
                if (QC < MAXV && v >= QC) continue; // solved where the walk meets it
                const float x[3] = {a.leaf.x[qx(e, v, 0)], a.leaf.x[qx(e, v, 1)], a.leaf.x[qx(e, v, 2)]};
                double q[3];
                exact_q(x, w, p0, DX, p0, plo, phi, tol, q);
                for (int i = 0; i < 3; ++i) AT(qs, 3 * v + i) = q[i];
            }
            moved += elem_bytes(nv) + 96; // the fragment and its image's vertices
        }
        double o[3], mom[10];
        unsigned e2 = 1;
        if (ok) {
            e2 = leaf_moments<QC>(nv, nbs, qs, c.mom_order, o, mom, a, e, t, lo);
            st |= e2;
        }
        if (ok && !e2 && mom[0] > 0.0) {
            const GridDev& g = *gp;
            if (gi < 0) {
                st |= ST_INDEX;
            } else {
                key = ((unsigned long long)gi << c.rec_ibits) | (unsigned long long)(t - c.rec_item_base);
                const double m0 = mom[0];
                double u[3];
                for (int i = 0; i < 3; ++i) u[i] = mom[1 + i] / m0;
                rec[0] = m0;
                for (int i = 0; i < 3; ++i) rec[1 + i] = o[i] + u[i];
                rec[4] = mom[4] / m0 - u[0] * u[0];
                rec[5] = mom[5] / m0 - u[0] * u[1];
                rec[6] = mom[6] / m0 - u[0] * u[2];
                rec[7] = mom[7] / m0 - u[1] * u[1];
                rec[8] = mom[8] / m0 - u[1] * u[2];
                rec[9] = mom[9] / m0 - u[2] * u[2];
                ++frags;
                verts += nv;
                if constexpr (INLINE) {
                    // atomic mode: straight into the voxel's sums, no record
                    const double f = c.acc.factor ? c.acc.factor[t] : 1.0;
                    accumulate_fragment(c, g, c.grids ? (int)c.it.grid[t] : 0, gi, lo, t, rec, f);
                } else {
                    has = true;
                }
                if (!c.acc.factor) atomicAdd(&a.vsum[t], m0);
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
                    if (k < c.rec_nmom) dst[k] = rec[k];
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

// FP32 walks can misplace a vertex that falls back to its FP32 position by
// ~1e-7 of the tet: each breadth-first image's fragment masses are scaled by
// target / (sum of its fragment q-volumes), so that it deposits exactly its
// mass inside the window.  init stores -target in scale (1, or the image's
// exact FP64 q-volume inside the window).  The deep-tree images (key KEY_DEEP)
// are not the walk's: their kernel, which may run beside this one, sets their
// scale itself.
__global__ void k_bfs_finalize(BfsArgs a, long long nitems)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nitems; t += (long long)gridDim.x * blockDim.x)
        if (a.c.it.key[t] < KEY_DEEP && a.c.scale[t] < 0.0)
            a.c.scale[t] = a.vsum[t] > 0.0 ? -a.c.scale[t] / a.vsum[t] : 1.0;
}

__global__ void k_bfs_advance(BfsArgs a) { ++*a.pass_idx; }

cudaError_t launch_bfs_advance(const BfsArgs& a, cudaStream_t s)
{
    k_bfs_advance<<<1, 1, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_bfs_finalize(const BfsArgs& a, long long nitems, int num_sms, cudaStream_t s)
{
    k_bfs_finalize<<<num_sms * 8, 256, 0, s>>>(a, nitems);
    return cudaGetLastError();
}

// ---- launchers ----

static constexpr size_t LEVEL_SMEM = 3 * MAXV * BB * sizeof(uint32_t); // links of the cut polyhedron and its children
// links of every vertex, FP64 q of the cached ones
static constexpr size_t LEAF_SMEM = MAXV * BB * sizeof(uint32_t) + 3 * MAXV * BB * sizeof(double);
static constexpr size_t LEAF_REC_SMEM = MAXV * BB * sizeof(uint32_t) + 3 * QC_REC * BB * sizeof(double);

// resident blocks per SM of each kernel (one full wave of grid-stride blocks)
static int g_blocks[4] = {0, 0, 0, 0};
static void occupancy();
void bfs_prepare() { occupancy(); }
void bfs_level_carveout(int percent)
{
    static int set = -1;
    if (percent == set) return;
    cudaFuncSetAttribute(k_bfs_level, cudaFuncAttributePreferredSharedMemoryCarveout, percent > 0 ? percent : -1);
    cudaGetLastError();
    set = percent;
}
static void occupancy()
{
    if (g_blocks[0]) return;
    cudaFuncSetAttribute(k_bfs_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LEVEL_SMEM);
    cudaFuncSetAttribute(k_bfs_leaf<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LEAF_SMEM);
    cudaFuncSetAttribute(k_bfs_leaf<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LEAF_REC_SMEM);
    int b[4] = {1, 1, 1, 1};
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b[0], k_bfs_init, BB, 0) != cudaSuccess) b[0] = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b[1], k_bfs_level, BB, LEVEL_SMEM) != cudaSuccess) b[1] = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b[2], k_bfs_leaf<true>, BB, LEAF_SMEM) != cudaSuccess)
        b[2] = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b[3], k_bfs_leaf<false>, BB, LEAF_REC_SMEM) != cudaSuccess)
        b[3] = 1;
    cudaGetLastError();
    for (int i = 0; i < 4; ++i) g_blocks[i] = b[i] > 0 ? b[i] : 1;
}

cudaError_t launch_bfs_init(const BfsArgs& a, int num_sms, cudaStream_t s)
{
    occupancy();
    k_bfs_init<<<num_sms * g_blocks[0], BB, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_bfs_level(const BfsArgs& a, int num_sms, cudaStream_t s)
{
    occupancy();
    // a.level_blocks (< the occupancy limit): fewer resident blocks, with the shared memory they
    // leave given to L1 (the positions the cut reads through the read-only cache)
    const int nb = (a.level_blocks > 0 && a.level_blocks < g_blocks[1]) ? a.level_blocks : g_blocks[1];
    k_bfs_level<<<num_sms * nb, BB, LEVEL_SMEM, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_bfs_leaf(const BfsArgs& a, int num_sms, cudaStream_t s)
{
    occupancy();
    if (a.c.acc.sum) k_bfs_leaf<true><<<num_sms * g_blocks[2], BB, LEAF_SMEM, s>>>(a);
    else k_bfs_leaf<false><<<num_sms * g_blocks[3], BB, LEAF_REC_SMEM, s>>>(a);
    return cudaGetLastError();
}

} // namespace psib
