// psib_clip.cuh -- the clip-and-deposit kernels (included by clip_fp64.cu and
// clip_mixed.cu, which compile it with and without FMA contraction).
//
// One thread voxelizes one tet image (psi_voxelize_tet, src/geometry.c:60-188):
// window clip and index box (src/geometry.c:806-843), bisection to voxels,
// moments, projection with the tet's deformation matrices, deposit.
//
// The grid fields of the reference are mass-weighted means and covariances
// built by a sequential online update (src/geometry.c:164-186), which atomics
// cannot reproduce.  The kernels therefore accumulate sums that merge exactly:
//   pass 1: W = sum w, SX = sum w (c_f - c_vox), SV = sum w v_f
//   pass 2: XX = sum w (S_f + (c_f - mu)(c_f - mu)^T), likewise XV, VV,
// with w = mass * m0 of a fragment, c_f its centroid, S_f its central second
// moment and mu the voxel mean from pass 1.  Centring on the voxel mean keeps
// the covariances free of cancellation; the finalize kernel merges them into
// the existing fields with the same parallel-axis rule as the online update.
// In record mode (deterministic, FP64) each fragment's raw q-moments are
// written out instead, to be applied per voxel in the reference's order.
#pragma once
#include "psib_device.cuh"
#include "psib_kernels.h"

namespace psib {

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

__device__ __forceinline__ void deposit(const ClipArgs& a, const TetFrame& F, double mass, const double* mom,
                                        long long gi, const int* vox)
{
    const AccDev& A = a.acc;
    const double w = mass * mom[0];
    double cm[3], cv[3];
    if (A.flags & (F_X | F_XX | F_XV)) centroid(mom, F.x0, F.DX, cm);
    if (A.flags & (F_V | F_XV | F_VV)) centroid(mom, F.v0, F.DV, cv);
    if (a.pass == 1) {
        atomicAdd(&A.W[gi], w);
        if (A.flags & F_X)
            for (int i = 0; i < 3; ++i) {
                const double c = a.g.w0[i] + a.g.d[i] * (vox[i] + 0.5);
                atomicAdd(&A.SX[3 * gi + i], w * (cm[i] - c));
            }
        if (A.flags & F_V)
            for (int i = 0; i < 3; ++i) atomicAdd(&A.SV[3 * gi + i], w * cv[i]);
        return;
    }
    double dx[3] = {0, 0, 0}, dv[3] = {0, 0, 0};
    if (A.flags & (F_XX | F_XV))
        for (int i = 0; i < 3; ++i) dx[i] = cm[i] - A.MX[3 * gi + i];
    if (A.flags & (F_XV | F_VV))
        for (int i = 0; i < 3; ++i) dv[i] = cv[i] - A.MV[3 * gi + i];
    double S[3][3];
    if (A.flags & F_XX) {
        second_moment(mom, F.x0, cm, F.DX, F.x0, cm, F.DX, F.x0, cm, F.x0, cm, S);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) atomicAdd(&A.XX[9 * gi + 3 * i + j], w * (S[i][j] + dx[i] * dx[j]));
    }
    if (A.flags & F_XV) {
        second_moment(mom, F.x0, cm, F.DX, F.v0, cv, F.DV, F.x0, cm, F.v0, cv, S);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) atomicAdd(&A.XV[9 * gi + 3 * i + j], w * (S[i][j] + dx[i] * dv[j]));
    }
    if (A.flags & F_VV) {
        second_moment(mom, F.v0, cv, F.DV, F.v0, cv, F.DV, F.v0, cv, F.v0, cv, S);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) atomicAdd(&A.VV[9 * gi + 3 * i + j], w * (S[i][j] + dv[i] * dv[j]));
    }
}

// Per-thread counters, folded into the global ones once per thread.
struct Tally {
    unsigned long long frags = 0, verts = 0, splits = 0;
};

// Voxelize item t.  S points to NS polyhedron slots owned by this thread.
template <class R, int NS, bool RECORD>
__device__ void clip_item(const ClipArgs& a, long long t, Poly<R>* S, unsigned& st, Tally& tally)
{
    const long long cap = a.it.cap;
    double p[4][3];
    for (int v = 0; v < 4; ++v)
        for (int i = 0; i < 3; ++i) p[v][i] = a.it.p[(3 * v + i) * cap + t];
    const double mass = a.it.mass[t];
    TetFrame F;
    for (int i = 0; i < 3; ++i) {
        F.x0[i] = p[0][i];
        for (int j = 0; j < 3; ++j) F.DX[i][j] = p[j + 1][i] - p[0][i];
    }
    if (a.acc.flags & (F_V | F_XV | F_VV)) {
        double u[4][3];
        for (int v = 0; v < 4; ++v)
            for (int i = 0; i < 3; ++i) u[v][i] = a.it.u[(3 * v + i) * cap + t];
        for (int i = 0; i < 3; ++i) {
            F.v0[i] = u[0][i];
            for (int j = 0; j < 3; ++j) F.DV[i][j] = u[j + 1][i] - u[0][i];
        }
    }
    double rb[2][3];
    aabb4(p, rb);

    // window planes n.x + d >= 0 and voxel index box (src/geometry.c:816-842)
    int pax[6], psg[6], npl = 0;
    double pdd[6];
    int lo[3], hi[3];
    for (int i = 0; i < 3; ++i) {
        double cmin = rb[0][i], cmax = rb[1][i];
        const bool clo = a.g.w0[i] > cmin, chi = a.g.w1[i] < cmax;
        if (clo) cmin = a.g.w0[i];
        if (chi) cmax = a.g.w1[i];
        if (clo) { pax[npl] = i; psg[npl] = 1; pdd[npl] = -cmin; npl++; }
        if (chi) { pax[npl] = i; psg[npl] = -1; pdd[npl] = cmax; npl++; }
        lo[i] = (int)floor((cmin - a.g.w0[i]) / a.g.d[i]);
        hi[i] = (int)ceil((cmax - a.g.w0[i]) / a.g.d[i]);
        if (lo[i] < 0) lo[i] = 0;
        if (hi[i] > a.g.n[i]) hi[i] = a.g.n[i];
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

    // Recentring for the FP32 kernel: coordinates relative to the index box's
    // lower corner, so FP32 keeps its precision at grid-cell scale.
    double org[3];
    for (int i = 0; i < 3; ++i) org[i] = (sizeof(R) == 8) ? 0.0 : a.g.w0[i] + a.g.d[i] * lo[i];

    int c;
    PSIB_ALLOC(c);
    R s[MAXV];
    // q-volume the fragments must add up to: 1 for a tet inside the window.
    double target = 1.0, msum = 0.0, mbest = -1.0;
    long long gbest = -1;
    if constexpr (sizeof(R) == 4) {
        if (npl > 0) {
            // The FP32 kernel clips against the window in FP64, so that a tet
            // split across periodic images still deposits exactly its mass.
            Poly<double> W[2];
            init_tet(W[0], p);
            double sd[MAXV];
            int cw = 0;
            for (int pl = 0; pl < npl && W[cw].nv > 0; ++pl) {
                const int ax = pax[pl];
                double smin = 1.0e30, smax = -1.0e30;
                uint32_t um = 0;
                for (int v = 0; v < W[cw].nv; ++v) {
                    double t0 = pdd[pl];
                    for (int i = 0; i < 3; ++i) t0 += W[cw].x[v][i] * (i == ax ? (double)psg[pl] : 0.0);
                    sd[v] = t0;
                    if (t0 < smin) smin = t0;
                    if (t0 > smax) smax = t0;
                    if (t0 < 0.0) um |= 1u << v;
                }
                if (smin >= 0.0) continue;
                if (smax <= 0.0) { W[cw].nv = 0; break; }
                const unsigned e = cut_poly<double, false>(W[cw], sd, um, W[1 - cw], W[1 - cw]);
                if (e) { st |= e; return; }
                cw = 1 - cw;
            }
            if (W[cw].nv == 0) return;
            double m0[10];
            const unsigned e = reduce_poly(W[cw], m0, 0);
            if (e) { st |= e; return; }
            target = m0[0];
            Poly<R>& P = S[c];
            P.nv = W[cw].nv;
            for (int v = 0; v < P.nv; ++v) {
                P.nb[v] = W[cw].nb[v];
                for (int i = 0; i < 3; ++i) {
                    P.x[v][i] = (R)(W[cw].x[v][i] - org[i]);
                    P.q[v][i] = (R)W[cw].q[v][i];
                }
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
        const R dd = (sizeof(R) == 8) ? (R)pdd[pl] : (R)(pdd[pl] + psg[pl] * org[ax]);
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
        const unsigned e = cut_poly<R, false>(P, s, um, S[o], S[o]);
        PSIB_FREE(c);
        c = o;
        if (e) { st |= e; return; }
    }
    for (int i = 0; i < 3; ++i) { S[c].lo[i] = lo[i]; S[c].hi[i] = hi[i]; }

    double mom[10];
    const int order = a.mom_order;
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
                // a single voxel: reduce and deposit (src/geometry.c:873-884)
                const unsigned e = reduce_poly(P, mom, order);
                if (e) { st |= e; return; }
                if (mom[0] > 0.0) {
                    if (P.lo[0] >= a.g.n[0] || P.lo[1] >= a.g.n[1] || P.lo[2] >= a.g.n[2]) {
                        st |= ST_INDEX;
                    } else {
                        const long long gi = ((long long)a.g.n[1] * P.lo[0] + P.lo[1]) * a.g.n[2] + P.lo[2];
                        tally.frags++;
                        tally.verts += P.nv;
                        if constexpr (sizeof(R) == 4) {
                            msum += mom[0];
                            if (mom[0] > mbest) { mbest = mom[0]; gbest = gi; }
                        }
                        if (RECORD) {
                            const unsigned long long r = atomicAdd(a.rec_n, 1ull);
                            if (r < a.rec_cap) {
                                a.rec_key[r] = ((unsigned long long)gi << 32) | (unsigned long long)(t - a.rec_item_base);
                                for (int k = 0; k < a.rec_nmom; ++k) a.rec_mom[r * a.rec_nmom + k] = mom[k];
                            } else {
                                st |= ST_RECORDS;
                            }
                        } else {
                            deposit(a, F, mass, mom, gi, P.lo);
                        }
                    }
                }
            } else {
                // split at the middle grid plane of the longest axis (src/geometry.c:886-893)
                tally.splits++;
                const double coord = a.g.d[ax] * (P.lo[ax] + dmax / 2) + a.g.w0[ax];
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
                    const unsigned e = cut_poly<R, true>(P, s, um, S[l], S[r]);
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
    if constexpr (sizeof(R) == 4) {
        // FP32 fragments miss the exact q-volume by O(1e-7); book the residual
        // on the largest fragment's voxel so the tet deposits exactly its mass.
        if (!RECORD && a.pass == 1 && gbest >= 0) atomicAdd(&a.acc.W[gbest], mass * (target - msum));
    }
#undef PSIB_ALLOC
#undef PSIB_FREE
}

// Persistent kernel: warps take 32 consecutive queue entries at a time.
template <class R, int NS, bool RECORD, bool SCRATCH>
__device__ __forceinline__ void clip_loop(const ClipArgs& a, Poly<R>* S)
{
    const int lane = threadIdx.x & 31;
    unsigned st = 0;
    Tally tally;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(a.head, 32ull);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= (unsigned long long)a.n) break;
        const long long i = (long long)base + lane;
        if (i < a.n) {
            const long long t = a.order ? (long long)a.order[a.order_base + i] : a.order_base + i;
            clip_item<R, NS, RECORD>(a, t, S, st, tally);
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
