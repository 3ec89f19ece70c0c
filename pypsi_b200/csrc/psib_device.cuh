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
// reference's fragment moments bit for bit.  R = float gives the walk of the
// mixed-precision kernel: FP32 positions, plane distances and cuts and no q
// at all; at each leaf the fragment's vertices are recomputed in FP64 from the
// planes they lie on (exact_vertices) and its moments taken in FP64.
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
    using real = R;
    using mask_t = uint32_t; // one bit per vertex
    static constexpr bool has_q = true;
    static constexpr int CAP = MAXV;
    R x[MAXV][3];      // position
    R q[MAXV][3];      // barycentric mass coordinate
    uint32_t nb[MAXV]; // neighbour links: bits 0-7, 8-15, 16-23; bits 24-30: plane tags
    int nv;
    int lo[3], hi[3];  // voxel index box
};

// The FP32 walk carries positions and links only (q is rebuilt at the leaf).
template <>
struct Poly<float> {
    using real = float;
    using mask_t = uint32_t;
    static constexpr bool has_q = false;
    static constexpr int CAP = MAXV;
    float x[MAXV][3];
    uint32_t nb[MAXV];
    int nv;
    int lo[3], hi[3];
};

// A fragment for the moment sums: FP64 q and links.
struct QPoly {
    static constexpr int CAP = MAXV;
    double q[MAXV][3];
    uint32_t nb[MAXV];
    int nv;
};

__device__ __forceinline__ int nbget(uint32_t w, int k) { return (w >> (8 * k)) & 0xFFu; }
__device__ __forceinline__ uint32_t nbset(uint32_t w, int k, int v)
{
    return (w & ~(0xFFu << (8 * k))) | ((uint32_t)v << (8 * k));
}
__device__ __forceinline__ int rank_in(uint32_t mask, int v) { return __popc(mask & ((1u << v) - 1u)); }
__device__ __forceinline__ int rank_in(uint64_t mask, int v) { return __popcll(mask & ((1ull << v) - 1ull)); }
__device__ __forceinline__ int popc_of(uint32_t m) { return __popc(m); }
__device__ __forceinline__ int popc_of(uint64_t m) { return __popcll(m); }

// Plane tags of a vertex, in the top byte of its link word.  Bit 24 + j: the
// vertex lies on the face of the original tet opposite its vertex j.  Bit
// 28 + a: it lies on a grid (or window) plane normal to axis a.  A cut vertex
// lies on the planes both ends of its edge lie on, plus the cutting plane, so
// a cut ANDs the two tags and adds the cut's axis.  Generic vertices carry
// exactly three tags.  The tags change no arithmetic: the adjoint uses them to
// find the fragment faces that move with the tet's vertices, and the mixed
// kernel to recompute each fragment vertex in FP64 from its three planes.
constexpr uint32_t TAG_MASK = 0x0F000000u;   // tet faces
constexpr uint32_t PLANE_MASK = 0x70000000u; // grid planes by axis
constexpr uint32_t ALL_TAGS = TAG_MASK | PLANE_MASK;
__device__ __forceinline__ uint32_t tags(uint32_t w) { return (w & TAG_MASK) >> 24; }
__device__ __forceinline__ uint32_t axis_tag(int ax) { return 0x10000000u << ax; }

// Close the cut face: each vertex created by a cut (index >= base) gets its
// two remaining links by walking around the face it opened
// (src/geometry.c:459-482, :646-669).
template <class PT>
__device__ __forceinline__ bool link_cut_vertices(PT& P, int base)
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
template <class PT, bool BOTH>
__device__ __forceinline__ unsigned cut_any(const PT& in, const typename PT::real* s, typename PT::mask_t umask, PT& lo,
                                            PT& up, uint32_t cut_tag)
{
    using R = typename PT::real;
    using M = typename PT::mask_t;
    constexpr int CAP = PT::CAP;
    static_assert(CAP < 8 * (int)sizeof(M), "a vertex mask bit for every vertex");
    const int n = in.nv;
    const M all = ((M)1 << n) - (M)1;
    const M lmask = all & ~umask;
    const int nl = popc_of(lmask), nu = popc_of(umask);
    for (int v = 0; v < n; ++v) {
        const bool u = (umask >> v) & 1u;
        if (!BOTH && u) continue;
        PT& o = u ? up : lo;
        const M sm = u ? umask : lmask;
        const int j = rank_in(sm, v);
        o.x[j][0] = in.x[v][0]; o.x[j][1] = in.x[v][1]; o.x[j][2] = in.x[v][2];
        if constexpr (PT::has_q) {
            o.q[j][0] = in.q[v][0]; o.q[j][1] = in.q[v][1]; o.q[j][2] = in.q[v][2];
        }
        const uint32_t w = in.nb[v];
        uint32_t ow = 0xFFFFFFu | (w & ALL_TAGS);
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
            if (nl + k >= CAP || (BOTH && nu + k >= CAP)) return ST_OVERFLOW;
            const R sc = s[vc], sn = s[vn];
            const R iw = R(1) / (sc - sn);
            R px[3], pq[3];
            for (int i = 0; i < 3; ++i) {
                px[i] = iw * (in.x[vn][i] * sc - in.x[vc][i] * sn);
                if constexpr (PT::has_q) pq[i] = iw * (in.q[vn][i] * sc - in.q[vc][i] * sn);
            }
            const int il = nl + k;
            const uint32_t tg = (w & in.nb[vn] & ALL_TAGS) | cut_tag;
            for (int i = 0; i < 3; ++i) {
                lo.x[il][i] = px[i];
                if constexpr (PT::has_q) lo.q[il][i] = pq[i];
            }
            lo.nb[il] = 0xFFFF00u | (uint32_t)jc | tg;
            lo.nb[jc] = nbset(lo.nb[jc], np, il);
            if (BOTH) {
                const int iu = nu + k;
                const int jn = rank_in(umask, vn);
                for (int i = 0; i < 3; ++i) {
                    up.x[iu][i] = px[i];
                    if constexpr (PT::has_q) up.q[iu][i] = pq[i];
                }
                up.nb[iu] = 0xFFFF00u | (uint32_t)jn | tg;
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

template <class R, bool BOTH>
__device__ __forceinline__ unsigned cut_poly(const Poly<R>& in, const R* s, uint32_t umask, Poly<R>& lo, Poly<R>& up,
                                             uint32_t cut_tag)
{
    return cut_any<Poly<R>, BOTH>(in, s, umask, lo, up, cut_tag);
}

// The tet as a vertex graph with q = (0, e_x, e_y, e_z) (src/geometry.c:769-804).
template <class PT, class T>
__device__ __forceinline__ void init_tet(PT& P, const T (*x)[3])
{
    P.nb[0] = 1u | (3u << 8) | (2u << 16);
    P.nb[1] = 2u | (3u << 8) | (0u << 16);
    P.nb[2] = 0u | (3u << 8) | (1u << 16);
    P.nb[3] = 1u | (2u << 8) | (0u << 16);
    for (int v = 0; v < 4; ++v) P.nb[v] |= (0xFu & ~(1u << v)) << 24;
    for (int v = 0; v < 4; ++v)
        for (int i = 0; i < 3; ++i) {
            P.x[v][i] = x[v][i];
            if constexpr (PT::has_q) P.q[v][i] = (v == i + 1) ? 1 : 0;
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
    // one bit per (vertex, link); at least two words, as the density path has always used
    constexpr int NW = (3 * PT::CAP + 63) / 64 > 2 ? (3 * PT::CAP + 63) / 64 : 2;
    uint64_t done[NW] = {};
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

// Adjoint of a fragment's mass fraction with respect to the tet's vertex
// positions.  The fraction is m0 = S(P) / S(T): the signed x-space volumes of
// the fragment and of the tet, both in the orientation of the q-space fan
// triangles.  When the tet's vertices move, only the fragment faces lying on
// the tet's own faces move (voxel and window planes stay put), a point p of
// such a face with velocity sum_i lambda_i(p) dx_i, so
//   dS(P)/dx_i = sum over those faces of the integral of lambda_i dN
//              = sum over their fan triangles of N lambda_i(centroid),
// with N = (p1 - p0) x (p2 - p0) / 2 and lambda = (1 - qx - qy - qz, qx, qy, qz).
// Adds g * dS(P)/dx_i to A[i].  A face lies on a tet face when all its vertices
// carry that face's tag.
template <class PT>
__device__ __forceinline__ unsigned adjoint_poly(const PT& P, double g, double (*A)[3])
{
    // one bit per (vertex, link); at least two words, as the density path has always used
    constexpr int NW = (3 * PT::CAP + 63) / 64 > 2 ? (3 * PT::CAP + 63) / 64 : 2;
    uint64_t done[NW] = {};
    for (int vs = 0; vs < P.nv; ++vs)
        for (int ks = 0; ks < 3; ++ks) {
            const int b0 = 3 * vs + ks;
            if ((done[b0 >> 6] >> (b0 & 63)) & 1ull) continue;
            done[b0 >> 6] |= 1ull << (b0 & 63);
            int vc = vs;
            int vn = nbget(P.nb[vc], ks);
            if (vn >= P.nv) return ST_GRAPH;
            uint32_t ft = tags(P.nb[vs]);
            uint32_t w = P.nb[vn];
            int k = (nbget(w, 0) == vc) ? 0 : (nbget(w, 1) == vc) ? 1 : (nbget(w, 2) == vc) ? 2 : 3;
            if (k == 3) return ST_GRAPH;
            vc = vn;
            int kn = (k + 1) % 3;
            int b = 3 * vc + kn;
            done[b >> 6] |= 1ull << (b & 63);
            ft &= tags(w);
            vn = nbget(P.nb[vc], kn);
            double ns[3] = {0.0, 0.0, 0.0}, nq[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
            int steps = 0;
            while (vn != vs) {
                if (++steps > WALK_CAP || vn >= P.nv) return ST_GRAPH;
                if (ft) {
                    double e1[3], e2[3], qc[3];
                    for (int i = 0; i < 3; ++i) {
                        e1[i] = (double)P.x[vn][i] - (double)P.x[vs][i];
                        e2[i] = (double)P.x[vc][i] - (double)P.x[vs][i];
                        qc[i] = ((double)P.q[vs][i] + (double)P.q[vn][i] + (double)P.q[vc][i]) * (1.0 / 3.0);
                    }
                    const double n[3] = {0.5 * (e1[1] * e2[2] - e1[2] * e2[1]), 0.5 * (e1[2] * e2[0] - e1[0] * e2[2]),
                                         0.5 * (e1[0] * e2[1] - e1[1] * e2[0])};
                    for (int i = 0; i < 3; ++i) {
                        ns[i] += n[i];
                        for (int j = 0; j < 3; ++j) nq[i][j] += n[i] * qc[j];
                    }
                }
                w = P.nb[vn];
                ft &= tags(w);
                k = (nbget(w, 0) == vc) ? 0 : (nbget(w, 1) == vc) ? 1 : (nbget(w, 2) == vc) ? 2 : 3;
                if (k == 3) return ST_GRAPH;
                vc = vn;
                kn = (k + 1) % 3;
                b = 3 * vc + kn;
                done[b >> 6] |= 1ull << (b & 63);
                vn = nbget(P.nb[vc], kn);
            }
            if (ft) {
                for (int i = 0; i < 3; ++i) {
                    A[0][i] += g * (ns[i] - nq[i][0] - nq[i][1] - nq[i][2]);
                    for (int j = 0; j < 3; ++j) A[1 + j][i] += g * nq[i][j];
                }
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

// Moments of a polyhedron about the q-space point o (order 0, 1 or 2): the
// same fan triangles as reduce_poly, with every vertex taken relative to o.
// With o on the polyhedron the cone volumes do not cancel and the first and
// second moments are fragment-sized, so central moments follow without
// cancellation.  Used by the mixed-precision kernel.
template <class PT>
__device__ __forceinline__ unsigned reduce_about(const PT& P, const double* o, double* mom, int order)
{
    for (int i = 0; i < 10; ++i) mom[i] = 0.0;
    // one bit per (vertex, link); at least two words, as the density path has always used
    constexpr int NW = (3 * PT::CAP + 63) / 64 > 2 ? (3 * PT::CAP + 63) / 64 : 2;
    uint64_t done[NW] = {};
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

// Recompute the vertices of an FP32 fragment in FP64 (mixed-precision kernel).
// Each vertex is the intersection of the three planes its tags name, solved in
// q-space: tet faces are q_j = 0 (j = 1..3) and qx + qy + qz = 1; the grid
// plane x_a = c is (DX q)_a = c - x0_a with DX[a][j] = x_{j+1,a} - x_{0,a}.  Of
// the two grid planes normal to axis a that bound the fragment's voxel
// ([plo_a, phi_a]), the vertex lies on the nearer.  An axis tag only says "on
// some plane normal to a": an edge from one such plane to another keeps the
// tag after the AND, so a tag is kept only when the vertex lies within tol_a of
// a bounding plane (FP32 positions are good to ~1e-5 of a voxel there).  The
// tags always include the vertex's true planes; of four, the grid plane
// farthest from the vertex is dropped.  A vertex whose tags do not name
// three planes, or whose planes are singular, gets q = DX^-1 (x - x0) from its
// FP32 position.  The links and tags are copied.
// Solve n_i . q = b_i (i = 0..2) by Cramer's rule; false when singular.
__device__ __forceinline__ bool solve3(const double (*n)[3], const double* b, double* q)
{
    const double c12[3] = {n[1][1] * n[2][2] - n[1][2] * n[2][1], n[1][2] * n[2][0] - n[1][0] * n[2][2],
                           n[1][0] * n[2][1] - n[1][1] * n[2][0]};
    const double c20[3] = {n[2][1] * n[0][2] - n[2][2] * n[0][1], n[2][2] * n[0][0] - n[2][0] * n[0][2],
                           n[2][0] * n[0][1] - n[2][1] * n[0][0]};
    const double c01[3] = {n[0][1] * n[1][2] - n[0][2] * n[1][1], n[0][2] * n[1][0] - n[0][0] * n[1][2],
                           n[0][0] * n[1][1] - n[0][1] * n[1][0]};
    const double det = n[0][0] * c12[0] + n[0][1] * c12[1] + n[0][2] * c12[2];
    if (!(det != 0.0) || !isfinite(det)) return false;
    const double id = 1.0 / det;
    for (int i = 0; i < 3; ++i) q[i] = (b[0] * c12[i] + b[1] * c20[i] + b[2] * c01[i]) * id;
    return true;
}

// Plane idx of a vertex's tags as a row n . q = b: idx 0..3 is the tet face
// opposite vertex idx (qx + qy + qz = 1, or q_{idx-1} = 0), idx 4..6 the grid
// plane x_a = pc_a (a = idx - 4), i.e. DX[a] . q = pc_a - p0_a.  Selects by
// value so that everything stays in registers.
__device__ __forceinline__ void plane_row(int idx, const double (*DX)[3], const double* pc, const double* p0,
                                          double* n, double& b)
{
    if (idx < 4) {
        n[0] = (idx == 0 || idx == 1) ? 1.0 : 0.0;
        n[1] = (idx == 0 || idx == 2) ? 1.0 : 0.0;
        n[2] = (idx == 0 || idx == 3) ? 1.0 : 0.0;
        b = idx == 0 ? 1.0 : 0.0;
    } else {
        const int a = idx - 4;
        for (int c = 0; c < 3; ++c) n[c] = a == 0 ? DX[0][c] : a == 1 ? DX[1][c] : DX[2][c];
        b = a == 0 ? pc[0] - p0[0] : a == 1 ? pc[1] - p0[1] : pc[2] - p0[2];
    }
}

// q of one vertex of an FP32 fragment: x is its FP32 position relative to org,
// w its link word (tags), DX the tet's edge matrix, p0 its vertex 0.
__device__ __forceinline__ void exact_q(const float* x, uint32_t w, const double* p0, const double (*DX)[3],
                                        const double* org, const double* plo, const double* phi, const double* tol,
                                        double* q)
{
    const uint32_t tf = (w >> 24) & 0xFu;
    uint32_t ap = 0;
    double pc[3], dist[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double xv = (double)x[a] + org[a];
        const double dl = fabs(xv - plo[a]), dh = fabs(xv - phi[a]);
        pc[a] = dl <= dh ? plo[a] : phi[a];
        dist[a] = dl <= dh ? dl : dh;
        if (((w >> (28 + a)) & 1u) && dist[a] <= tol[a]) ap |= 1u << a;
    }
    // a vertex near the edge or corner of its voxel can keep a fourth tag:
    // the tet-face tags are exact, so drop the grid plane farthest in units of tol
    while (__popc(tf) + __popc(ap) > 3) {
        int far = -1;
        double df = -1.0;
#pragma unroll
        for (int a = 0; a < 3; ++a)
            if (((ap >> a) & 1u) && dist[a] / tol[a] > df) { far = a; df = dist[a] / tol[a]; }
        if (far < 0) break;
        ap &= ~(1u << far);
    }
    double n0[3], n1[3], n2[3], b0, b1, b2;
    bool ok = __popc(tf) + __popc(ap) == 3;
    if (ok) {
        uint32_t m = tf | (ap << 4);
        const int i0 = __ffs(m) - 1;
        m &= m - 1;
        const int i1 = __ffs(m) - 1;
        m &= m - 1;
        const int i2 = __ffs(m) - 1;
        plane_row(i0, DX, pc, p0, n0, b0);
        plane_row(i1, DX, pc, p0, n1, b1);
        plane_row(i2, DX, pc, p0, n2, b2);
        const double nn[3][3] = {{n0[0], n0[1], n0[2]}, {n1[0], n1[1], n1[2]}, {n2[0], n2[1], n2[2]}};
        const double bb[3] = {b0, b1, b2};
        ok = solve3(nn, bb, q);
    }
    if (!ok) {
        // position -> q through the tet's own map: rows DX[a], right side x_a - x0_a
        const double bb[3] = {((double)x[0] + org[0]) - p0[0], ((double)x[1] + org[1]) - p0[1],
                              ((double)x[2] + org[2]) - p0[2]};
        if (!solve3(DX, bb, q)) q[0] = q[1] = q[2] = 0.0; // a flat tet: its fragments have no volume
    }
}

__device__ __forceinline__ void exact_vertices(const Poly<float>& P, const double (*p)[3], const double* org,
                                               const double* plo, const double* phi, const double* tol,
                                               QPoly& Q)
{
    double DX[3][3];
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 3; ++j) DX[a][j] = p[j + 1][a] - p[0][a];
    Q.nv = P.nv;
    for (int v = 0; v < P.nv; ++v) {
        Q.nb[v] = P.nb[v];
        exact_q(P.x[v], P.nb[v], p[0], DX, org, plo, phi, tol, Q.q[v]);
    }
}

} // namespace psib
