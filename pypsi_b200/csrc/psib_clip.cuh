// psib_clip.cuh -- the clip kernels (included by clip_fp64.cu and
// clip_mixed.cu, which compile it without and with FMA contraction).
//
// One thread voxelizes one tet image (psi_voxelize_tet, src/geometry.c:60-188):
// window clip and index box (src/geometry.c:806-843), depth-first bisection to
// single voxels (:852-896), q-space moments of each fragment (:692-767).  Each
// fragment becomes a record -- key (voxel, image) and up to ten moments --
// and nothing is accumulated here.  The records are then sorted by key and
// each voxel's run is applied to the grid fields in the reference's order by
// one thread (apply kernels in tess.cu), which reproduces the reference's
// online field update (src/geometry.c:164-186) exactly: no atomics, one clip
// pass for every field order.
//
// Records of the FP64 kernel hold the reference's raw moments m0..m9 about
// q = 0.  Records of the FP32 kernel hold m0, the fragment's q-centroid and its
// central q-space second moment (moments taken about a vertex of the fragment,
// reduce_about), which keep FP32 vertex errors from being amplified; its
// threads also store each image's mass-correction factor (exact FP64 volume of
// the window-clipped tet over the sum of its FP32 fragment volumes).
//
// Each thread owns a contiguous region of a global scratch buffer for its
// polyhedron slots: contiguous per-thread storage keeps every 32-byte sector a
// thread touches full of its own data, where the compiler's local memory would
// interleave threads word by word and waste most of each sector as soon as
// threads index different slots.
#pragma once
#include "psib_accum.cuh"
#include "psib_adjoint.cuh"
#include "psib_device.cuh"
#include "psib_kernels.h"

namespace psib {

// Per-thread scratch region: NS polyhedron slots, then (FP32 kernels) the
// FP64 leaf fragment and two FP64 polyhedra for the window clip.  Every part
// starts on a 16-byte boundary.
__host__ __device__ constexpr size_t round16(size_t b) { return (b + 15) & ~(size_t)15; }

template <class R, int NS>
__host__ __device__ constexpr size_t leaf_offset() { return round16(sizeof(Poly<R>) * NS); }

template <class R, int NS>
__host__ __device__ constexpr size_t wclip_offset() { return leaf_offset<R, NS>() + round16(sizeof(QPoly)); }

template <class R, int NS>
__host__ __device__ constexpr size_t region_bytes()
{
    return sizeof(R) == 4 ? wclip_offset<R, NS>() + round16(2 * sizeof(Poly<double>)) : leaf_offset<R, NS>();
}

__device__ __forceinline__ void aabb4(const double (*p)[3], double (*rb)[3])
{
    for (int i = 0; i < 3; ++i) {
        rb[0][i] = 1.0e30;
        rb[1][i] = -1.0e30;
    }
    for (int v = 0; v < 4; ++v)
        for (int i = 0; i < 3; ++i) {
            if (p[v][i] < rb[0][i]) rb[0][i] = p[v][i];
            if (p[v][i] > rb[1][i]) rb[1][i] = p[v][i];
        }
}

// Per-thread counters, folded into the global ones once per thread.
struct Tally {
    unsigned long long frags = 0, verts = 0, splits = 0;
};

// One fragment of image t in voxel lo (global gi) of grid g: a record, or in
// the atomic mode (central records only) straight into the voxel's sums.
__device__ __forceinline__ void write_record(const ClipArgs& a, const GridDev& g, long long gi, const int* lo,
                                             long long t, const double* mom, unsigned& st)
{
    if (a.acc.sum) {
        accumulate_fragment(a, g, a.grids ? (int)a.it.grid[t] : 0, gi, lo, t, mom,
                            a.acc.factor ? a.acc.factor[t] : 1.0);
        return;
    }
    // one atomic per group of lanes that reach this point together: the record
    // counter is a single address that every fragment of the launch hits
    const unsigned act = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(act) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(a.rec_n, (unsigned long long)__popc(act));
    base = __shfl_sync(act, base, leader);
    const unsigned long long r = base + __popc(act & ((1u << lane) - 1u));
    if (r < a.rec_cap) {
        a.rec_key[r] = ((unsigned long long)gi << a.rec_ibits) | (unsigned long long)(t - a.rec_item_base);
        double* dst = a.rec_mom + r * a.rec_nmom;
        for (int k = 0; k < a.rec_nmom; ++k) dst[k] = mom[k];
    } else {
        st |= ST_RECORDS;
    }
}

// Voxelize item t.  S points to NS polyhedron slots owned by this thread;
// FP32 kernel only: QL to the FP64 leaf fragment, WC to two FP64 polyhedra.  CENTRAL: write centroid-form
// records (always so in the FP32 kernel; the FP64 kernel does it when it
// serves the mixed-precision mode).  ADJ (FP64 only): instead of writing
// records, pull the upstream gradient of the m field back to the positions of
// the image's four particles (and to its element's mass).  FULL (with ADJ):
// the gradient of every field, through the per-voxel coefficients adj_coef
// (psib_adjoint.cuh), back to positions, velocities and masses.
// The particles a tet vertex of image t moves with: its own particle (pid >= 0, weight 1), or for
// a vertex of a refined element (pid a refine_vertex_code) the element's nodes with their
// interpolation weights at the vertex's place -- trilinear for 8-node, triquadratic (Lagrange on
// 0, 1/2, 1 per axis) for 27-node elements, as the refinement interpolates.  f(id, weight) for each
// with a nonzero weight; false on an id out of range.
template <class F>
__device__ bool for_vertex_sources(const ClipArgs& a, int pid, long long e, F&& f)
{
    if (pid >= 0) {
        if (pid >= a.adj_npart) return false;
        f(pid, 1.0);
        return true;
    }
    if (pid == -1) return false;
    int x[3], lvl;
    refine_vertex_decode(pid, x, lvl);
    const MeshDev& m = a.adj_mesh;
    const int et = m.elemtype;
    if ((et != 8 && et != 27) || e < 0 || e >= m.nelem) return false;
    const int nb = et == 27 ? 3 : 2;
    double b[3][3];
    for (int i = 0; i < 3; ++i) {
        const double u = x[i] * (1.0 / 128);
        if (et == 27) {
            b[i][0] = 2.0 * (u - 0.5) * (u - 1.0);
            b[i][1] = 4.0 * u * (1.0 - u);
            b[i][2] = 2.0 * u * (u - 0.5);
        } else {
            b[i][0] = 1.0 - u;
            b[i][1] = u;
        }
    }
    long long nyz = 0;
    int ei = 0, ej = 0, ek = 0;
    if (!m.conn) {
        nyz = (long long)m.edim[1] * m.edim[2];
        ei = (int)(e / nyz);
        ej = (int)((e / m.edim[2]) % m.edim[1]);
        ek = (int)(e % m.edim[2]);
    }
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j)
            for (int k = 0; k < nb; ++k) {
                const double w = b[0][i] * b[1][j] * b[2][k];
                if (w == 0.0) continue;
                long long id;
                if (m.conn) {
                    id = m.conn[e * et + (et == 27 ? 9 * i + 3 * j + k : 4 * i + 2 * j + k)];
                } else { // implicit block connectivity (src/PSI.c:644-656)
                    id = (long long)m.bdim[1] * m.bdim[2] * ((ei + i) % m.bdim[0]) +
                         (long long)m.bdim[2] * ((ej + j) % m.bdim[1]) + ((ek + k) % m.bdim[2]);
                }
                if (id < 0 || id >= a.adj_npart) return false;
                f((int)id, w);
            }
    return true;
}

// Tet mass / element mass of image t: the unrefined factor times 1/8 per refinement level.
__device__ __forceinline__ double image_mass_factor(const ClipArgs& a, long long t)
{
    const int pid = a.it.pid[t];
    if (pid > -2) return a.adj_mass_factor;
    int x[3], lvl;
    refine_vertex_decode(pid, x, lvl);
    double f = a.adj_mass_factor;
    for (int l = 0; l < lvl; ++l) f *= 0.125;
    return f;
}

template <class R, int NS, bool CENTRAL, bool ADJ = false, bool FULL = false>
__device__ void clip_item(const ClipArgs& a, long long t, Poly<R>* S, QPoly* QL, Poly<double>* WC, unsigned& st,
                          Tally& tally)
{
    static_assert(!ADJ || (sizeof(R) == 8 && !CENTRAL), "the adjoint walks the FP64 fragments");
    static_assert(!FULL || ADJ, "FULL is a form of the adjoint");
    // the image's grid: its cutout's in a batch, whose voxels start at vbase
    const GridDev& g = a.grids ? a.grids[a.it.grid[t]] : a.g;
    const unsigned long long vbase = a.voff ? a.voff[a.it.grid[t]] : 0ull;
    const double* fr = a.it.frame + t * FRAME;
    double p[4][3];
    for (int v = 0; v < 4; ++v)
        for (int i = 0; i < 3; ++i) p[v][i] = fr[3 * v + i];
    double rb[2][3];
    aabb4(p, rb);

    // window planes n.x + d >= 0 and voxel index box (src/geometry.c:816-842)
    int pax[6], psg[6], npl = 0;
    double pdd[6];
    int lo[3], hi[3];
    for (int i = 0; i < 3; ++i) {
        double cmin = rb[0][i], cmax = rb[1][i];
        const bool clo = g.w0[i] > cmin, chi = g.w1[i] < cmax;
        if (clo) cmin = g.w0[i];
        if (chi) cmax = g.w1[i];
        if (clo) { pax[npl] = i; psg[npl] = 1; pdd[npl] = -cmin; npl++; }
        if (chi) { pax[npl] = i; psg[npl] = -1; pdd[npl] = cmax; npl++; }
        lo[i] = (int)floor((cmin - g.w0[i]) / g.d[i]);
        hi[i] = (int)ceil((cmax - g.w0[i]) / g.d[i]);
        if (lo[i] < 0) lo[i] = 0;
        if (hi[i] > g.n[i]) hi[i] = g.n[i];
    }

    // slot pool
    uint64_t freem = (NS >= 64) ? ~0ull : ((1ull << NS) - 1ull);
    int8_t stk[NS];
    int top = 0;
#define PSIB_ALLOC(dst)                                            \
    {                                                              \
        const int _i = __ffsll((long long)freem) - 1;              \
        if (_i < 0) { st |= ST_OVERFLOW; return; }                 \
        freem &= ~(1ull << _i);                                    \
        dst = _i;                                                  \
    }
#define PSIB_FREE(i) (freem |= 1ull << (i))

    // Recentring for the FP32 kernel: coordinates relative to the tet's first
    // vertex, so FP32 keeps its precision at the scale of the tet (which can be
    // far smaller than a voxel once refined).
    double org[3];
    for (int i = 0; i < 3; ++i) org[i] = (sizeof(R) == 8) ? 0.0 : p[0][i];

    int c;
    PSIB_ALLOC(c);
    R s[MAXV];
    double target = 1.0, vsum = 0.0; // exact and FP32 q-volume of the image (FP32 kernel)
    if constexpr (sizeof(R) == 4) {
        if (npl > 0) {
            // The FP32 kernel clips against the window in FP64, so that a tet
            // split across periodic images still deposits exactly its mass.
            Poly<double>* W[2] = {&WC[0], &WC[1]};
            init_tet(*W[0], p);
            double sd[MAXV];
            int cw = 0;
            for (int pl = 0; pl < npl && W[cw]->nv > 0; ++pl) {
                const int ax = pax[pl];
                double smin = 1.0e30, smax = -1.0e30;
                uint32_t um = 0;
                for (int v = 0; v < W[cw]->nv; ++v) {
                    double t0 = pdd[pl];
                    for (int i = 0; i < 3; ++i) t0 += W[cw]->x[v][i] * (i == ax ? (double)psg[pl] : 0.0);
                    sd[v] = t0;
                    if (t0 < smin) smin = t0;
                    if (t0 > smax) smax = t0;
                    if (t0 < 0.0) um |= 1u << v;
                }
                if (smin >= 0.0) continue;
                if (smax <= 0.0) { W[cw]->nv = 0; break; }
                const unsigned e = cut_poly<double, false>(*W[cw], sd, um, *W[1 - cw], *W[1 - cw], axis_tag(ax));
                if (e) { st |= e; return; }
                cw = 1 - cw;
            }
            if (W[cw]->nv == 0) { a.scale[t] = 1.0; return; }
            double m0[10];
            const unsigned e = reduce_poly(*W[cw], m0, 0);
            if (e) { st |= e; return; }
            target = m0[0];
            Poly<R>& P = S[c];
            const Poly<double>& Q = *W[cw];
            P.nv = Q.nv;
            for (int v = 0; v < P.nv; ++v) {
                P.nb[v] = Q.nb[v];
                for (int i = 0; i < 3; ++i) P.x[v][i] = (R)(Q.x[v][i] - org[i]);
            }
        }
    }
    if (sizeof(R) == 8 || npl == 0) {
        R xr[4][3];
        for (int v = 0; v < 4; ++v)
            for (int i = 0; i < 3; ++i) xr[v][i] = (sizeof(R) == 8) ? (R)p[v][i] : (R)(p[v][i] - org[i]);
        init_tet(S[c], xr);
    }
    if (sizeof(R) == 4) npl = 0; // the FP32 kernel has clipped against the window above
    // window clip (src/geometry.c:391-501), one plane at a time
    for (int pl = 0; pl < npl && S[c].nv > 0; ++pl) {
        Poly<R>& P = S[c];
        const int ax = pax[pl];
        const R sg = (R)psg[pl];
        const R dd = (R)pdd[pl];
        R smin = (R)1.0e30, smax = (R)-1.0e30;
        uint32_t um = 0;
        for (int v = 0; v < P.nv; ++v) {
            // ((d + x0 n0) + x1 n1) + x2 n2 with n = +-e_ax
            R t0 = dd;
            for (int i = 0; i < 3; ++i) t0 += P.x[v][i] * (i == ax ? sg : (R)0);
            s[v] = t0;
            if (t0 < smin) smin = t0;
            if (t0 > smax) smax = t0;
            if (t0 < (R)0) um |= 1u << v;
        }
        if (smin >= (R)0) continue;
        if (smax <= (R)0) { P.nv = 0; break; }
        int o;
        PSIB_ALLOC(o);
        const unsigned e = cut_poly<R, false>(P, s, um, S[o], S[o], axis_tag(ax));
        PSIB_FREE(c);
        c = o;
        if (e) { st |= e; return; }
    }
    for (int i = 0; i < 3; ++i) { S[c].lo[i] = lo[i]; S[c].hi[i] = hi[i]; }

    double mom[10];
    const int order = a.mom_order;
    // adjoint accumulators: sum over fragments of g dS(P)/dx_i, and of g m0
    double A[4][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    double B = 0.0;
    // full adjoint: the image's frame and its accumulators
    AdjItem T;
    AdjAcc acc;
    if constexpr (FULL) {
        for (int i = 0; i < 3; ++i) {
            T.x0[i] = p[0][i];
            T.v0[i] = fr[FR_U + i];
            for (int j = 0; j < 3; ++j) {
                T.DX[i][j] = p[j + 1][i] - p[0][i];
                T.DV[i][j] = fr[FR_U + 3 * (j + 1) + i] - fr[FR_U + i];
            }
        }
        T.mass = fr[FR_MASS];
        adj_zero(acc);
    }
    for (;;) {
        Poly<R>& P = S[c];
        bool done_node = true;
        if (P.nv > 0) {
            int dmax = 0, ax = 0;
            for (int i = 0; i < 3; ++i) {
                const int sz = P.hi[i] - P.lo[i];
                if (sz > dmax) { dmax = sz; ax = i; }
            }
            if (dmax <= 1) {
                // a single voxel (src/geometry.c:873-884)
                double o[3] = {0.0, 0.0, 0.0};
                if constexpr (CENTRAL && sizeof(R) == 8)
                    for (int i = 0; i < 3; ++i) o[i] = (double)P.q[0][i];
                if constexpr (sizeof(R) == 4) {
                    // the FP32 walk fixed the fragment's graph; its vertices are
                    // recomputed in FP64 from their planes before the moments
                    double plo[3], phi[3], tol[3];
                    for (int i = 0; i < 3; ++i) {
                        plo[i] = g.d[i] * P.lo[i] + g.w0[i];
                        phi[i] = g.d[i] * (P.lo[i] + 1) + g.w0[i];
                        tol[i] = 1.0e-3 * g.d[i];
                    }
                    exact_vertices(P, p, org, plo, phi, tol, *QL);
                    for (int i = 0; i < 3; ++i) o[i] = QL->q[0][i];
                }
                double gv = 0.0;
                const double* cf = nullptr;
                if constexpr (ADJ) {
                    if (P.lo[0] < g.n[0] && P.lo[1] < g.n[1] && P.lo[2] < g.n[2]) {
                        const long long vi = ((long long)g.n[1] * P.lo[0] + P.lo[1]) * g.n[2] + P.lo[2];
                        if constexpr (FULL) {
                            cf = a.adj_coef + vi * ADJ_NCOEF;
                            gv = 1.0; // every fragment is walked: the forward's voxels all hold mass
                        } else {
                            gv = a.adj_gm[vi];
                        }
                    }
                }
                unsigned e;
                if constexpr (FULL) e = reduce_poly(P, mom, 2);
                else if constexpr (ADJ) e = gv != 0.0 ? reduce_poly(P, mom, 0) : 0u;
                else if constexpr (sizeof(R) == 4) e = reduce_about(*QL, o, mom, order);
                else e = CENTRAL ? reduce_about(P, o, mom, order) : reduce_poly(P, mom, order);
                if (e) { st |= e; return; }
                if (ADJ && gv == 0.0) {
                    // no upstream gradient in this voxel: nothing to pull back
                } else if (mom[0] > 0.0) {
                    if (P.lo[0] >= g.n[0] || P.lo[1] >= g.n[1] || P.lo[2] >= g.n[2]) {
                        st |= ST_INDEX;
                    } else {
                        const long long gi =
                            (long long)vbase + ((long long)g.n[1] * P.lo[0] + P.lo[1]) * g.n[2] + P.lo[2];
                        tally.frags++;
                        tally.verts += P.nv;
                        if constexpr (FULL) {
                            const unsigned e2 = adjoint_fragment(P, mom, cf, T, acc);
                            if (e2) { st |= e2; return; }
                        } else if constexpr (ADJ) {
                            const unsigned e2 = adjoint_poly(P, gv, A);
                            if (e2) { st |= e2; return; }
                            B += gv * mom[0];
                        } else if constexpr (CENTRAL) {
                            // m0, q-centroid, central q second moment (xx xy xz yy yz zz)
                            vsum += mom[0];
                            double rec[10];
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
                            write_record(a, g, gi, P.lo, t, rec, st);
                        } else {
                            write_record(a, g, gi, P.lo, t, mom, st);
                        }
                    }
                }
            } else {
                // split at the middle grid plane of the longest axis (src/geometry.c:886-893)
                tally.splits++;
                const double coord = g.d[ax] * (P.lo[ax] + dmax / 2) + g.w0[ax];
                const R cr = (sizeof(R) == 8) ? (R)coord : (R)(coord - org[ax]);
                uint32_t um = 0;
                for (int v = 0; v < P.nv; ++v) {
                    s[v] = cr - P.x[v][ax];
                    if (s[v] < (R)0) um |= 1u << v;
                }
                const int nlo = dmax / 2, nup = dmax - dmax / 2;
                if (um == 0) {
                    P.hi[ax] -= nup; // everything below the plane: keep the lower half in place
                    done_node = false;
                } else if (um == (1u << P.nv) - 1u) {
                    P.lo[ax] += nlo;
                    done_node = false;
                } else {
                    int l, r;
                    PSIB_ALLOC(l);
                    PSIB_ALLOC(r);
                    const unsigned e = cut_poly<R, true>(P, s, um, S[l], S[r], axis_tag(ax));
                    if (e) { st |= e; return; }
                    for (int i = 0; i < 3; ++i) {
                        S[l].lo[i] = P.lo[i]; S[l].hi[i] = P.hi[i];
                        S[r].lo[i] = P.lo[i]; S[r].hi[i] = P.hi[i];
                    }
                    S[l].hi[ax] -= nup;
                    S[r].lo[ax] += nlo;
                    PSIB_FREE(c);
                    if (top >= NS) { st |= ST_OVERFLOW; return; }
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
    if constexpr (FULL) {
        // dL/dp_k = (mass / vol) * surface integrals - (dvol/dp_k / vol) * I0 - (grad v)^T J_k, plus the
        // quirk's explicit term on the first vertex; dL/du_k = J_k (plus its velocity term); dL/dmass = I0 / mass
        double e[3][3];
        for (int v = 0; v < 3; ++v)
            for (int i = 0; i < 3; ++i) e[v][i] = p[v + 1][i] - p[0][i];
        double dS[4][3];
        for (int v = 0; v < 3; ++v) {
            const double* u = e[(v + 1) % 3];
            const double* w = e[(v + 2) % 3];
            dS[v + 1][0] = (u[1] * w[2] - u[2] * w[1]) * (1.0 / 6.0);
            dS[v + 1][1] = (u[2] * w[0] - u[0] * w[2]) * (1.0 / 6.0);
            dS[v + 1][2] = (u[0] * w[1] - u[1] * w[0]) * (1.0 / 6.0);
        }
        for (int i = 0; i < 3; ++i) dS[0][i] = -(dS[1][i] + dS[2][i] + dS[3][i]);
        const double sT = e[0][0] * dS[1][0] + e[0][1] * dS[1][1] + e[0][2] * dS[1][2];
        if (sT != 0.0) {
            // grad v = DV DX^-1: solve DX^T G^T = DV^T row by row (DX^-1 = adj(DX)^T / det)
            double inv[3][3];
            {
                const double(*D)[3] = T.DX;
                const double det = D[0][0] * (D[1][1] * D[2][2] - D[1][2] * D[2][1]) -
                                   D[0][1] * (D[1][0] * D[2][2] - D[1][2] * D[2][0]) +
                                   D[0][2] * (D[1][0] * D[2][1] - D[1][1] * D[2][0]);
                const double id = 1.0 / det;
                inv[0][0] = (D[1][1] * D[2][2] - D[1][2] * D[2][1]) * id;
                inv[0][1] = (D[0][2] * D[2][1] - D[0][1] * D[2][2]) * id;
                inv[0][2] = (D[0][1] * D[1][2] - D[0][2] * D[1][1]) * id;
                inv[1][0] = (D[1][2] * D[2][0] - D[1][0] * D[2][2]) * id;
                inv[1][1] = (D[0][0] * D[2][2] - D[0][2] * D[2][0]) * id;
                inv[1][2] = (D[0][2] * D[1][0] - D[0][0] * D[1][2]) * id;
                inv[2][0] = (D[1][0] * D[2][1] - D[1][1] * D[2][0]) * id;
                inv[2][1] = (D[0][1] * D[2][0] - D[0][0] * D[2][1]) * id;
                inv[2][2] = (D[0][0] * D[1][1] - D[0][1] * D[1][0]) * id;
            }
            double gvel[3][3]; // d v_c / d x_a
            for (int c2 = 0; c2 < 3; ++c2)
                for (int a2 = 0; a2 < 3; ++a2)
                    gvel[c2][a2] = T.DV[c2][0] * inv[0][a2] + T.DV[c2][1] * inv[1][a2] + T.DV[c2][2] * inv[2][a2];
            const double rho = T.mass / sT;
            for (int v = 0; v < 4; ++v) {
                double gp[3], gu[3];
                for (int i = 0; i < 3; ++i) {
                    gp[i] = rho * acc.bnd[v][i] - dS[v][i] / sT * acc.I0;
                    for (int c2 = 0; c2 < 3; ++c2) gp[i] -= gvel[c2][i] * acc.J[v][c2];
                    gu[i] = acc.J[v][i];
                    if (v == 0) {
                        gp[i] += acc.qa[i];
                        gu[i] += acc.qb[i];
                    }
                }
                const bool ok = for_vertex_sources(a, a.it.pid[v * a.it.cap + t], a.it.elem[t], [&](int id, double w) {
                    for (int i = 0; i < 3; ++i) {
                        atomicAdd(&a.adj_gpos[3 * (long long)id + i], w * gp[i]);
                        if (a.adj_gvel) atomicAdd(&a.adj_gvel[3 * (long long)id + i], w * gu[i]);
                    }
                });
                if (!ok) st |= ST_INDEX;
            }
            if (a.adj_gmass && T.mass != 0.0)
                atomicAdd(&a.adj_gmass[a.it.elem[t]], acc.I0 / T.mass * image_mass_factor(a, t));
        }
    } else if constexpr (ADJ) {
        // d m0 / dx_i = (dS(P)/dx_i - m0 dS(T)/dx_i) / S(T), times the image's mass
        if (B != 0.0 || A[0][0] != 0.0 || A[0][1] != 0.0 || A[0][2] != 0.0 || A[1][0] != 0.0 || A[1][1] != 0.0 ||
            A[1][2] != 0.0 || A[2][0] != 0.0 || A[2][1] != 0.0 || A[2][2] != 0.0 || A[3][0] != 0.0 ||
            A[3][1] != 0.0 || A[3][2] != 0.0) {
            double e[3][3];
            for (int v = 0; v < 3; ++v)
                for (int i = 0; i < 3; ++i) e[v][i] = p[v + 1][i] - p[0][i];
            double dS[4][3];
            for (int v = 0; v < 3; ++v) {
                const double* u = e[(v + 1) % 3];
                const double* w = e[(v + 2) % 3];
                dS[v + 1][0] = (u[1] * w[2] - u[2] * w[1]) * (1.0 / 6.0);
                dS[v + 1][1] = (u[2] * w[0] - u[0] * w[2]) * (1.0 / 6.0);
                dS[v + 1][2] = (u[0] * w[1] - u[1] * w[0]) * (1.0 / 6.0);
            }
            for (int i = 0; i < 3; ++i) dS[0][i] = -(dS[1][i] + dS[2][i] + dS[3][i]);
            const double sT = e[0][0] * dS[1][0] + e[0][1] * dS[1][1] + e[0][2] * dS[1][2];
            const double mass = fr[FR_MASS];
            if (sT != 0.0) {
                const double f = mass / sT;
                for (int v = 0; v < 4; ++v) {
                    const bool ok = for_vertex_sources(a, a.it.pid[v * a.it.cap + t], a.it.elem[t], [&](int id, double w) {
                        for (int i = 0; i < 3; ++i)
                            atomicAdd(&a.adj_gpos[3 * (long long)id + i], w * f * (A[v][i] - B * dS[v][i]));
                    });
                    if (!ok) st |= ST_INDEX;
                }
            }
            if (a.adj_gmass) atomicAdd(&a.adj_gmass[a.it.elem[t]], B * image_mass_factor(a, t));
        }
    }
    if constexpr (sizeof(R) == 4) {
        // FP32 fragments miss the exact q-volume by O(1e-7): the apply kernel
        // scales this image's fragment masses by target / vsum.
        a.scale[t] = vsum > 0.0 ? target / vsum : 1.0;
    } else if constexpr (CENTRAL) {
        a.scale[t] = 1.0;
    }
#undef PSIB_ALLOC
#undef PSIB_FREE
}

// Persistent kernel body: warps take 32 consecutive queue entries at a time.
template <class R, int NS, bool CENTRAL, bool ADJ = false, bool FULL = false>
__device__ __forceinline__ void clip_loop(const ClipArgs& a)
{
    const int lane = threadIdx.x & 31;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    char* region = (char*)a.scratch + tid * region_bytes<R, NS>();
    Poly<R>* S = (Poly<R>*)region;
    QPoly* QL = (QPoly*)(region + leaf_offset<R, NS>());
    Poly<double>* WC = (Poly<double>*)(region + wclip_offset<R, NS>());
    unsigned st = 0;
    Tally tally;
    const long long n = a.n_dev ? (long long)*a.n_dev : a.n;
    const long long ob = a.base_dev ? (long long)*a.base_dev : a.order_base;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(a.head, 32ull);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= (unsigned long long)n) break;
        const long long i = (long long)base + lane;
        if (i < n) {
            const long long t = a.order ? (long long)a.order[ob + i] : ob + i;
            clip_item<R, NS, CENTRAL, ADJ, FULL>(a, t, S, QL, WC, st, tally);
        }
    }
    if (st) atomicOr(a.status, st);
    if (a.counters) {
        atomicAdd(&a.counters[0], tally.frags);
        atomicAdd(&a.counters[1], tally.verts);
        atomicAdd(&a.counters[2], tally.splits);
    }
}

} // namespace psib
