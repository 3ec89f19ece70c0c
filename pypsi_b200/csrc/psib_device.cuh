// psib_device.cuh -- device-side geometry of the voxelizer.
//
// A tet image is cut into voxel fragments by recursive bisection of its voxel
// index box, as PyPSI's psi_voxels_next does (src/geometry.c:852-896): split the
// longest axis of the box at its middle grid plane until the box is one voxel,
// then integrate the fragment's polynomial moments in barycentric "mass
// coordinates" q (src/geometry.c:692-767).  One CUDA thread owns one tet image.
//
// Polyhedra live in fixed-size slots (MAXV vertices, 3 byte-sized neighbour
// links packed in one word).  A slot free-mask replaces the reference's copying
// stack of 64 polyhedra: a split writes its two halves into free slots, the
// lower half is parked on a small index stack and the upper half is processed
// next, which is the reference's visiting order.
//
// The split and clip produce the same vertex order as the reference (surviving
// vertices in order, then cut vertices in creation order), and the moment sums
// run over the same fan triangles in the same order.  Compiled without FMA
// contraction (--fmad=false) and with R = double this reproduces the
// reference's fragment moments bit for bit; R = float gives the mixed-precision
// kernel (FP32 plane distances and interpolation, FP64 moments).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace psib {

constexpr int MAXV = 20;       // vertices of one polyhedron; <= 10 faces bound it by 16
constexpr int DMAX_MAIN = 8;   // bisection depth served by the main clip kernel
constexpr int NS_MAIN = DMAX_MAIN + 3;
constexpr int DMAX_BIG = 40;   // deeper trees go to the big-tet kernel
constexpr int SPAN_MAX = 16;   // longer index boxes also go to it (FP64 in both precisions)
constexpr int NS_BIG = DMAX_BIG + 3;
constexpr int WALK_CAP = 64;   // a face has < MAXV edges; longer walks mean a broken graph

// status bits written by kernels (atomicOr); the host maps them to PSIB_ERR_*
enum : unsigned {
    ST_OVERFLOW = 1u,  // polyhedron outgrew MAXV or the slot pool
    ST_GRAPH = 2u,     // a face walk did not close
    ST_INDEX = 4u,     // voxel or particle index out of range
    ST_RECORDS = 8u,   // fragment record buffer full (deterministic mode)
    ST_DEPTH = 16u,    // tet image deeper than the big-tet kernel supports
};

template <class R>
struct Poly {
    R x[MAXV][3];      // position
    R q[MAXV][3];      // barycentric mass coordinate
    uint32_t nb[MAXV]; // neighbour links: bits 0-7, 8-15, 16-23
    int nv;
    int lo[3], hi[3];  // voxel index box
};

__device__ __forceinline__ int nbget(uint32_t w, int k) { return (w >> (8 * k)) & 0xFFu; }
__device__ __forceinline__ uint32_t nbset(uint32_t w, int k, int v)
{
    return (w & ~(0xFFu << (8 * k))) | ((uint32_t)v << (8 * k));
}
__device__ __forceinline__ int rank_in(uint32_t mask, int v) { return __popc(mask & ((1u << v) - 1u)); }

// Close the cut face: each vertex created by a cut (index >= base) gets its
// two remaining links by walking around the face it opened
// (src/geometry.c:459-482, :646-669).
template <class R>
__device__ __forceinline__ bool link_cut_vertices(Poly<R>& P, int base)
{
    for (int vs = base; vs < P.nv; ++vs) {
        int vc = vs, vn = nbget(P.nb[vs], 0);
        int steps = 0;
        do {
            if (vn >= P.nv) return false;
            uint32_t w = P.nb[vn];
            int k = (nbget(w, 0) == vc) ? 0 : (nbget(w, 1) == vc) ? 1 : (nbget(w, 2) == vc) ? 2 : 3;
            if (k == 3 || ++steps > WALK_CAP) return false;
            vc = vn;
            vn = nbget(P.nb[vc], (k + 1) % 3);
        } while (vc < base);
        P.nb[vs] = nbset(P.nb[vs], 2, vc);
        P.nb[vc] = nbset(P.nb[vc], 1, vs);
    }
    return true;
}

// Cut `in` with per-vertex signed distances s[] (vertex v is on the upper side
// when bit v of umask is set, i.e. s[v] < 0).  Writes the lower side (s >= 0)
// to `lo` and, when BOTH, the upper side to `up`.  The cut vertex on edge
// (a lower, b upper) is (b*s_a - a*s_b) / (s_a - s_b) in the reference's
// operation order (src/geometry.c:441-445, :601-605).
template <class R, bool BOTH>
__device__ __forceinline__ unsigned cut_poly(const Poly<R>& in, const R* s, uint32_t umask, Poly<R>& lo, Poly<R>& up)
{
    const int n = in.nv;
    const uint32_t all = (1u << n) - 1u;
    const uint32_t lmask = all & ~umask;
    const int nl = __popc(lmask), nu = __popc(umask);
    for (int v = 0; v < n; ++v) {
        const bool u = (umask >> v) & 1u;
        if (!BOTH && u) continue;
        Poly<R>& o = u ? up : lo;
        const uint32_t sm = u ? umask : lmask;
        const int j = rank_in(sm, v);
        o.x[j][0] = in.x[v][0]; o.x[j][1] = in.x[v][1]; o.x[j][2] = in.x[v][2];
        o.q[j][0] = in.q[v][0]; o.q[j][1] = in.q[v][1]; o.q[j][2] = in.q[v][2];
        const uint32_t w = in.nb[v];
        uint32_t ow = 0xFFFFFFu;
        for (int k = 0; k < 3; ++k) {
            const int t = nbget(w, k);
            if (t >= n) return ST_GRAPH;
            if ((((umask >> t) & 1u) != 0) == u) ow = nbset(ow, k, rank_in(sm, t));
        }
        o.nb[j] = ow;
    }
    int k = 0;
    for (int vc = 0; vc < n; ++vc) {
        if ((umask >> vc) & 1u) continue;
        const uint32_t w = in.nb[vc];
        const int jc = rank_in(lmask, vc);
        for (int np = 0; np < 3; ++np) {
            const int vn = nbget(w, np);
            if (vn >= n) return ST_GRAPH;
            if (!((umask >> vn) & 1u)) continue;
            if (nl + k >= MAXV || (BOTH && nu + k >= MAXV)) return ST_OVERFLOW;
            const R sc = s[vc], sn = s[vn];
            const R iw = R(1) / (sc - sn);
            R px[3], pq[3];
            for (int i = 0; i < 3; ++i) {
                px[i] = iw * (in.x[vn][i] * sc - in.x[vc][i] * sn);
                pq[i] = iw * (in.q[vn][i] * sc - in.q[vc][i] * sn);
            }
            const int il = nl + k;
            for (int i = 0; i < 3; ++i) { lo.x[il][i] = px[i]; lo.q[il][i] = pq[i]; }
            lo.nb[il] = 0xFFFF00u | (uint32_t)jc;
            lo.nb[jc] = nbset(lo.nb[jc], np, il);
            if (BOTH) {
                const int iu = nu + k;
                const int jn = rank_in(umask, vn);
                for (int i = 0; i < 3; ++i) { up.x[iu][i] = px[i]; up.q[iu][i] = pq[i]; }
                up.nb[iu] = 0xFFFF00u | (uint32_t)jn;
                const uint32_t wn = in.nb[vn];
                const int kb = (nbget(wn, 0) == vc) ? 0 : (nbget(wn, 1) == vc) ? 1 : (nbget(wn, 2) == vc) ? 2 : 3;
                if (kb == 3) return ST_GRAPH;
                up.nb[jn] = nbset(up.nb[jn], kb, iu);
            }
            ++k;
        }
    }
    lo.nv = nl + k;
    if (!link_cut_vertices(lo, nl)) return ST_GRAPH;
    if (BOTH) {
        up.nv = nu + k;
        if (!link_cut_vertices(up, nu)) return ST_GRAPH;
    }
    return 0;
}

// The tet as a vertex graph with q = (0, e_x, e_y, e_z) (src/geometry.c:769-804).
template <class PT, class T>
__device__ __forceinline__ void init_tet(PT& P, const T (*x)[3])
{
    P.nb[0] = 1u | (3u << 8) | (2u << 16);
    P.nb[1] = 2u | (3u << 8) | (0u << 16);
    P.nb[2] = 0u | (3u << 8) | (1u << 16);
    P.nb[3] = 1u | (2u << 8) | (0u << 16);
    for (int v = 0; v < 4; ++v)
        for (int i = 0; i < 3; ++i) {
            P.x[v][i] = x[v][i];
            P.q[v][i] = (v == i + 1) ? 1 : 0;
        }
    P.nv = 4;
}

// Fragment moments in q-space: order 0 (1 value), 1 (4) or 2 (10), by fan
// triangles of every face, accumulated in the reference's order
// (src/geometry.c:692-767).  Always FP64.
template <class PT>
__device__ __forceinline__ unsigned reduce_poly(const PT& P, double* mom, int order)
{
    for (int i = 0; i < 10; ++i) mom[i] = 0.0;
    uint64_t done[2] = {0ull, 0ull};
    for (int vs = 0; vs < P.nv; ++vs)
        for (int ks = 0; ks < 3; ++ks) {
            const int b0 = 3 * vs + ks;
            if ((done[b0 >> 6] >> (b0 & 63)) & 1ull) continue;
            int vc = vs, kn = ks;
            done[b0 >> 6] |= 1ull << (b0 & 63);
            int vn = nbget(P.nb[vc], kn);
            if (vn >= P.nv) return ST_GRAPH;
            const double q0x = (double)P.q[vc][0], q0y = (double)P.q[vc][1], q0z = (double)P.q[vc][2];
            uint32_t w = P.nb[vn];
            int k = (nbget(w, 0) == vc) ? 0 : (nbget(w, 1) == vc) ? 1 : (nbget(w, 2) == vc) ? 2 : 3;
            vc = vn;
            kn = (k + 1) % 3;
            int b = 3 * vc + kn;
            done[b >> 6] |= 1ull << (b & 63);
            vn = nbget(P.nb[vc], kn);
            int steps = 0;
            while (vn != vs) {
                if (++steps > WALK_CAP || vn >= P.nv || k == 3) return ST_GRAPH;
                const double q1x = (double)P.q[vn][0], q1y = (double)P.q[vn][1], q1z = (double)P.q[vn][2];
                const double q2x = (double)P.q[vc][0], q2y = (double)P.q[vc][1], q2z = (double)P.q[vc][2];
                const double m = (-q2x * q1y * q0z + q1x * q2y * q0z + q2x * q0y * q1z
                                  - q0x * q2y * q1z - q1x * q0y * q2z + q0x * q1y * q2z);
                mom[0] += m;
                if (order > 0) {
                    mom[1] += 0.25 * m * (q0x + q1x + q2x);
                    mom[2] += 0.25 * m * (q0y + q1y + q2y);
                    mom[3] += 0.25 * m * (q0z + q1z + q2z);
                }
                if (order > 1) {
                    mom[4] += 0.1 * m * (q0x * q0x + q1x * q1x + q2x * q2x + q1x * q2x + q0x * (q1x + q2x));
                    mom[5] += 0.05 * m * (q2x * q0y + q2x * q1y + 2 * q2x * q2y + q0x * (2 * q0y + q1y + q2y) + q1x * (q0y + 2 * q1y + q2y));
                    mom[6] += 0.05 * m * (q2x * q0z + q2x * q1z + 2 * q2x * q2z + q0x * (2 * q0z + q1z + q2z) + q1x * (q0z + 2 * q1z + q2z));
                    mom[7] += 0.1 * m * (q0y * q0y + q1y * q1y + q2y * q2y + q1y * q2y + q0y * (q1y + q2y));
                    mom[8] += 0.05 * m * (q2y * q0z + q2y * q1z + 2 * q2y * q2z + q0y * (2 * q0z + q1z + q2z) + q1y * (q0z + 2 * q1z + q2z));
                    mom[9] += 0.1 * m * (q0z * q0z + q1z * q1z + q2z * q2z + q1z * q2z + q0z * (q1z + q2z));
                }
                w = P.nb[vn];
                k = (nbget(w, 0) == vc) ? 0 : (nbget(w, 1) == vc) ? 1 : (nbget(w, 2) == vc) ? 2 : 3;
                vc = vn;
                kn = (k + 1) % 3;
                if (k == 3) return ST_GRAPH;
                b = 3 * vc + kn;
                done[b >> 6] |= 1ull << (b & 63);
                vn = nbget(P.nb[vc], kn);
            }
        }
    return 0;
}

// ---- per-fragment projection to physical moments (src/geometry.c:81-161) ----

struct TetFrame {
    double x0[3], v0[3];
    double DX[3][3], DV[3][3]; // columns: vertex j+1 minus vertex 0
};

__device__ __forceinline__ void centroid(const double* mom, const double* o, const double (*D)[3], double* c)
{
    for (int i = 0; i < 3; ++i) {
        double t = mom[0] * o[i];
        for (int j = 0; j < 3; ++j) t += mom[j + 1] * D[i][j];
        c[i] = t / mom[0];
    }
}

// Central second moment of a fragment, the reference's expansion.  For the
// mixed x-v moment the reference pairs D_a with (o_a - c_a) in both cross
// terms (src/geometry.c:137-146); `cross` reproduces that with (oa, ca) on the
// first and (ob, cb) on the second cross term.
__device__ __forceinline__ void second_moment(const double* mom, const double* oa, const double* ca,
                                              const double (*Da)[3], const double* ob, const double* cb,
                                              const double (*Db)[3], const double* xa, const double* xca,
                                              const double* xb, const double* xcb, double (*S)[3])
{
    const int qi[3][3] = {{4, 5, 6}, {5, 7, 8}, {6, 8, 9}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double t = mom[0] * (oa[i] - ca[i]) * (ob[j] - cb[j]);
            for (int a = 0; a < 3; ++a) {
                t += Da[i][a] * mom[1 + a] * (xa[j] - xca[j]);
                t += Db[j][a] * mom[1 + a] * (xb[i] - xcb[i]);
            }
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) t += Da[i][a] * Db[j][b] * mom[qi[a][b]];
            S[i][j] = t / mom[0];
        }
}

} // namespace psib

namespace psib {

// ---- one-sided cuts for the per-voxel path kernels ----
//
// A lane follows the bisection path from the tet's index box down to its own
// voxel and keeps only the side of each split that contains that voxel.  The
// kept half of a split is the same polyhedron, vertex for vertex, that the
// reference's two-sided split produces for that child, so the fragment at the
// end of the path equals the reference's bit for bit.

constexpr int CAPV = 32; // vertex buffer of an in-place cut: kept vertices + cut vertices

template <class R>
struct Buf {
    R x[CAPV][3];
    R q[CAPV][3];
    uint32_t nb[CAPV];
    int nv;
};

__device__ __forceinline__ uint32_t low_mask(int n) { return n >= 32 ? 0xFFFFFFFFu : ((1u << n) - 1u); }

// Keep the lower side (s >= 0, keep_upper == false) or the upper side (s < 0)
// of a cut, in place.  The result lists the kept old vertices in order, then
// the cut vertices in the reference's creation order (lower vertex ascending,
// link ascending), exactly like the corresponding output of the two-sided
// split (src/geometry.c:593-690) or of the window clip (:436-500).
template <class R>
__device__ __forceinline__ unsigned half_cut(Buf<R>& P, const R* s, uint32_t umask, bool keep_upper)
{
    const int n = P.nv;
    const uint32_t lmask = low_mask(n) & ~umask;
    const uint32_t kmask = keep_upper ? umask : lmask;
    int nv = n;
    for (int vc = 0; vc < n; ++vc) {
        if (!((lmask >> vc) & 1u)) continue;
        for (int np = 0; np < 3; ++np) {
            const int vn = nbget(P.nb[vc], np);
            if (vn >= n) return ST_GRAPH; // lower-vertex links are only rewritten after they are read
            if (!((umask >> vn) & 1u)) continue;
            if (nv >= CAPV) return ST_OVERFLOW;
            const R sc = s[vc], sn = s[vn];
            const R iw = R(1) / (sc - sn);
            for (int i = 0; i < 3; ++i) {
                P.x[nv][i] = iw * (P.x[vn][i] * sc - P.x[vc][i] * sn);
                P.q[nv][i] = iw * (P.q[vn][i] * sc - P.q[vc][i] * sn);
            }
            if (!keep_upper) {
                P.nb[nv] = 0xFFFF00u | (uint32_t)vc;
                P.nb[vc] = nbset(P.nb[vc], np, nv);
            } else {
                P.nb[nv] = 0xFFFF00u | (uint32_t)vn;
                const uint32_t wn = P.nb[vn];
                const int kb = (nbget(wn, 0) == vc) ? 0 : (nbget(wn, 1) == vc) ? 1 : (nbget(wn, 2) == vc) ? 2 : 3;
                if (kb == 3) return ST_GRAPH;
                P.nb[vn] = nbset(wn, kb, nv);
            }
            ++nv;
        }
    }
    // close the cut face, walking the kept side (src/geometry.c:459-482)
    for (int vs = n; vs < nv; ++vs) {
        int vc = vs, vn = nbget(P.nb[vs], 0);
        int steps = 0;
        do {
            if (vn >= nv) return ST_GRAPH;
            const uint32_t w = P.nb[vn];
            const int k = (nbget(w, 0) == vc) ? 0 : (nbget(w, 1) == vc) ? 1 : (nbget(w, 2) == vc) ? 2 : 3;
            if (k == 3 || ++steps > WALK_CAP) return ST_GRAPH;
            vc = vn;
            vn = nbget(P.nb[vc], (k + 1) % 3);
        } while (vc < n);
        P.nb[vs] = nbset(P.nb[vs], 2, vc);
        P.nb[vc] = nbset(P.nb[vc], 1, vs);
    }
    // compact: kept old vertices, then the cut vertices, with links renumbered
    const int nk = __popc(kmask);
    for (int v = 0; v < nv; ++v) {
        const bool keep = v >= n || ((kmask >> v) & 1u);
        if (!keep) continue;
        const int dst = v < n ? rank_in(kmask, v) : nk + (v - n);
        uint32_t w = P.nb[v], ow = 0;
        for (int k = 0; k < 3; ++k) {
            const int t = nbget(w, k);
            const int tt = t < n ? rank_in(kmask, t) : nk + (t - n);
            ow |= (uint32_t)tt << (8 * k);
        }
        for (int i = 0; i < 3; ++i) {
            P.x[dst][i] = P.x[v][i];
            P.q[dst][i] = P.q[v][i];
        }
        P.nb[dst] = ow;
    }
    P.nv = nk + (nv - n);
    return 0;
}

// Moments of a polyhedron about the q-space point o (order 0, 1 or 2): the
// same fan triangles as reduce_poly, with every vertex taken relative to o.
// With o on the polyhedron the cone volumes do not cancel and the first and
// second moments are fragment-sized, so central moments follow without
// cancellation.  Used by the mixed-precision kernel.
template <class PT>
__device__ __forceinline__ unsigned reduce_about(const PT& P, const double* o, double* mom, int order)
{
    for (int i = 0; i < 10; ++i) mom[i] = 0.0;
    uint64_t done[2] = {0ull, 0ull};
    for (int vs = 0; vs < P.nv; ++vs)
        for (int ks = 0; ks < 3; ++ks) {
            const int b0 = 3 * vs + ks;
            if ((done[b0 >> 6] >> (b0 & 63)) & 1ull) continue;
            int vc = vs, kn = ks;
            done[b0 >> 6] |= 1ull << (b0 & 63);
            int vn = nbget(P.nb[vc], kn);
            if (vn >= P.nv) return ST_GRAPH;
            const double q0x = (double)P.q[vc][0] - o[0], q0y = (double)P.q[vc][1] - o[1], q0z = (double)P.q[vc][2] - o[2];
            uint32_t w = P.nb[vn];
            int k = (nbget(w, 0) == vc) ? 0 : (nbget(w, 1) == vc) ? 1 : (nbget(w, 2) == vc) ? 2 : 3;
            vc = vn;
            kn = (k + 1) % 3;
            int b = 3 * vc + kn;
            done[b >> 6] |= 1ull << (b & 63);
            vn = nbget(P.nb[vc], kn);
            int steps = 0;
            while (vn != vs) {
                if (++steps > WALK_CAP || vn >= P.nv || k == 3) return ST_GRAPH;
                const double q1x = (double)P.q[vn][0] - o[0], q1y = (double)P.q[vn][1] - o[1], q1z = (double)P.q[vn][2] - o[2];
                const double q2x = (double)P.q[vc][0] - o[0], q2y = (double)P.q[vc][1] - o[1], q2z = (double)P.q[vc][2] - o[2];
                const double m = (-q2x * q1y * q0z + q1x * q2y * q0z + q2x * q0y * q1z
                                  - q0x * q2y * q1z - q1x * q0y * q2z + q0x * q1y * q2z);
                mom[0] += m;
                if (order > 0) {
                    mom[1] += 0.25 * m * (q0x + q1x + q2x);
                    mom[2] += 0.25 * m * (q0y + q1y + q2y);
                    mom[3] += 0.25 * m * (q0z + q1z + q2z);
                }
                if (order > 1) {
                    mom[4] += 0.1 * m * (q0x * q0x + q1x * q1x + q2x * q2x + q1x * q2x + q0x * (q1x + q2x));
                    mom[5] += 0.05 * m * (q2x * q0y + q2x * q1y + 2 * q2x * q2y + q0x * (2 * q0y + q1y + q2y) + q1x * (q0y + 2 * q1y + q2y));
                    mom[6] += 0.05 * m * (q2x * q0z + q2x * q1z + 2 * q2x * q2z + q0x * (2 * q0z + q1z + q2z) + q1x * (q0z + 2 * q1z + q2z));
                    mom[7] += 0.1 * m * (q0y * q0y + q1y * q1y + q2y * q2y + q1y * q2y + q0y * (q1y + q2y));
                    mom[8] += 0.05 * m * (q2y * q0z + q2y * q1z + 2 * q2y * q2z + q0y * (2 * q0z + q1z + q2z) + q1y * (q0z + 2 * q1z + q2z));
                    mom[9] += 0.1 * m * (q0z * q0z + q1z * q1z + q2z * q2z + q1z * q2z + q0z * (q1z + q2z));
                }
                w = P.nb[vn];
                k = (nbget(w, 0) == vc) ? 0 : (nbget(w, 1) == vc) ? 1 : (nbget(w, 2) == vc) ? 2 : 3;
                if (k == 3) return ST_GRAPH;
                vc = vn;
                kn = (k + 1) % 3;
                b = 3 * vc + kn;
                done[b >> 6] |= 1ull << (b & 63);
                vn = nbget(P.nb[vc], kn);
            }
        }
    return 0;
}

} // namespace psib
