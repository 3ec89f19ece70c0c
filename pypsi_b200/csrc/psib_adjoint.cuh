// psib_adjoint.cuh -- the adjoint of every grid field (m, x, v, xx, xv, vv)
// with respect to particle positions, velocities and element masses.
//
// The fields a deposit leaves in a zeroed grid are functions of per-voxel sums
// over its fragments f (src/geometry.c:106-186 merges them one at a time;
// the merge is exact in these terms):
//   M = sum m_f,  X = sum P_f / M,  V = sum Q_f / M,
//   XX = (1/M) integral of rho (x - X)(x - X)^T,  VV alike,
//   XV = (1/M) [integral of rho (x - X)(v - V)^T + sum_f q_f],
// where rho = mass_T / vol_T is a tet's mass density, m_f, P_f, Q_f the
// integrals of rho, rho x, rho v over the fragment, v(x) the velocity
// interpolated linearly over the tet, and q_f = m_f (2 a b^T - a a^T - b b^T)
// with a = x_0 - P_f / m_f, b = v_0 - Q_f / m_f the reference's pairing of the
// x-v cross terms with the tet's first vertex (src/geometry.c:137-146).
//
// A first variation of the mass density at a point (x, v) of a voxel changes
// the loss L by phi(x, v) per unit mass, with (k_adj_coeffs, tess.cu)
//   phi = gM + gX.(x - X)/M + gV.(v - V)/M + <gXX, (x-X)(x-X)^T - XX>/M
//       + <gVV, (v-V)(v-V)^T - VV>/M + <gXV, (x-X)(v-V)^T - XV>/M,
// g* being dL/d(field) in the voxel: a quadratic in (x, v) about the voxel's
// means, so that nothing cancels.  The fragment's q_f adds, by the chain rule
// through (m_f, P_f, Q_f), phi_q = base + (dh/dP).(x - c) + (dh/dQ).(v - c_v)
// with c, c_v the fragment's centroids, and explicit terms on its tet's first
// vertex.  With the fragment's q-space moments (reduce_poly, order 2) every
// volume integral of a quadratic in (x, v) is exact:
//   dL/du_k   += integral of rho lambda_k dphi/dv                 (u: velocities)
//   dL/dmass  += integral of rho phi / mass_T
//   dL/dp_k   += rho * (surface integral of phi lambda_k over the fragment's
//                faces on the tet's faces, which move with the vertices; voxel
//                and window planes stay put)
//              - (dvol_T/dp_k / vol_T) integral of rho phi   (rho = mass / vol)
//              - (grad v)^T integral of rho lambda_k dphi/dv   (v(x) at fixed x)
// lambda being the barycentric coordinates of the tet.  The surface integrand
// is cubic; each fan triangle is integrated exactly by the degree-3 rule with
// weights 1/20 at the corners, 2/15 at the edge midpoints and 9/20 at the
// centroid.
#pragma once
#include "psib_device.cuh"

namespace psib {

constexpr int ADJ_NCOEF = 40; // per voxel: c0, cx[3], cv[3], A[9], B[9], C[9], X[3], V[3]

// The per-image constants of the adjoint walk.
struct AdjItem {
    double x0[3], v0[3], DX[3][3], DV[3][3]; // DX[i][j] = x_{j+1,i} - x_{0,i}
    double mass;
};

// Per-image accumulators (summed over the image's fragments).
struct AdjAcc {
    double bnd[4][3]; // surface integrals of phi lambda_k dN
    double J[4][3];   // integrals of rho lambda_k dphi/dv
    double I0;        // integral of rho phi
    double qa[3], qb[3]; // explicit quirk terms on the first vertex (position, velocity)
};

__device__ __forceinline__ void adj_zero(AdjAcc& c)
{
    for (int k = 0; k < 4; ++k)
        for (int i = 0; i < 3; ++i) c.bnd[k][i] = c.J[k][i] = 0.0;
    c.I0 = 0.0;
    for (int i = 0; i < 3; ++i) c.qa[i] = c.qb[i] = 0.0;
}

// A voxel's quadratic plus a fragment's linear quirk term, evaluated at (x, v).
struct AdjPhi {
    const double* cf; // the voxel's ADJ_NCOEF coefficients
    double base, hP[3], hQ[3], c[3], cv[3];
    __device__ __forceinline__ double operator()(const double* x, const double* v) const
    {
        double dx[3], dv[3];
        for (int i = 0; i < 3; ++i) {
            dx[i] = x[i] - cf[34 + i];
            dv[i] = v[i] - cf[37 + i];
        }
        double r = cf[0];
        for (int i = 0; i < 3; ++i) r += cf[1 + i] * dx[i] + cf[4 + i] * dv[i];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                r += dx[i] * cf[7 + 3 * i + j] * dx[j] + dv[i] * cf[16 + 3 * i + j] * dv[j] +
                     dx[i] * cf[25 + 3 * i + j] * dv[j];
        r += base;
        for (int i = 0; i < 3; ++i) r += hP[i] * (x[i] - c[i]) + hQ[i] * (v[i] - cv[i]);
        return r;
    }
};

// The adjoint contributions of one FP64 fragment P (its vertices' x and q) in
// a voxel with coefficients cf, whose q-space moments (order 2) are mom.
template <class PT>
__device__ __forceinline__ unsigned adjoint_fragment(const PT& P, const double* mom, const double* cf,
                                                     const AdjItem& T, AdjAcc& acc)
{
    const double m0 = mom[0];
    if (!(m0 > 0.0)) return 0;
    const double m1[3] = {mom[1], mom[2], mom[3]};
    const double M2[3][3] = {{mom[4], mom[5], mom[6]}, {mom[5], mom[7], mom[8]}, {mom[6], mom[8], mom[9]}};
    const double* Ac = cf + 7;
    const double* Bc = cf + 16;
    const double* Cc = cf + 25;
    // the fragment's mass and centroids
    const double m = T.mass * m0;
    double c[3], cv[3];
    for (int i = 0; i < 3; ++i) {
        c[i] = T.x0[i] + (T.DX[i][0] * m1[0] + T.DX[i][1] * m1[1] + T.DX[i][2] * m1[2]) / m0;
        cv[i] = T.v0[i] + (T.DV[i][0] * m1[0] + T.DV[i][1] * m1[1] + T.DV[i][2] * m1[2]) / m0;
    }
    // the quirk h = <C, m (2 a b^T - a a^T - b b^T)>, a = x0 - c, b = v0 - cv
    AdjPhi phi;
    phi.cf = cf;
    {
        double a[3], b[3];
        for (int i = 0; i < 3; ++i) {
            a[i] = T.x0[i] - c[i];
            b[i] = T.v0[i] - cv[i];
        }
        double base = 0.0, ha[3], hb[3];
        for (int i = 0; i < 3; ++i) {
            double sa = 0.0, sb = 0.0;
            for (int j = 0; j < 3; ++j) {
                const double cij = Cc[3 * i + j], cji = Cc[3 * j + i];
                base += cij * (2.0 * a[i] * b[j] - a[i] * a[j] - b[i] * b[j]);
                sa += 2.0 * cij * b[j] - (cij + cji) * a[j];
                sb += 2.0 * cji * a[j] - (cij + cji) * b[j];
            }
            ha[i] = m * sa;
            hb[i] = m * sb;
        }
        phi.base = base;
        for (int i = 0; i < 3; ++i) {
            phi.hP[i] = -ha[i] / m;
            phi.hQ[i] = -hb[i] / m;
            phi.c[i] = c[i];
            phi.cv[i] = cv[i];
            acc.qa[i] += ha[i];
            acc.qb[i] += hb[i];
        }
    }
    // phi(x(q), v(q)) = f0 + f1.q + q^T F2 q with x = x0 + DX q, v = v0 + DV q
    double al[3], be[3];
    for (int i = 0; i < 3; ++i) {
        al[i] = T.x0[i] - cf[34 + i];
        be[i] = T.v0[i] - cf[37 + i];
    }
    const double f0 = phi(T.x0, T.v0);
    // gradients of phi in x and v at q = 0
    double gx[3], gv[3];
    for (int i = 0; i < 3; ++i) {
        gx[i] = cf[1 + i] + phi.hP[i];
        gv[i] = cf[4 + i] + phi.hQ[i];
        for (int j = 0; j < 3; ++j) {
            gx[i] += (Ac[3 * i + j] + Ac[3 * j + i]) * al[j] + Cc[3 * i + j] * be[j];
            gv[i] += (Bc[3 * i + j] + Bc[3 * j + i]) * be[j] + Cc[3 * j + i] * al[j];
        }
    }
    double f1[3], F2[3][3];
    for (int j = 0; j < 3; ++j) {
        f1[j] = 0.0;
        for (int i = 0; i < 3; ++i) f1[j] += T.DX[i][j] * gx[i] + T.DV[i][j] * gv[i];
    }
    for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) {
            double s = 0.0;
            for (int i = 0; i < 3; ++i)
                for (int l = 0; l < 3; ++l)
                    s += T.DX[i][j] * Ac[3 * i + l] * T.DX[l][k] + T.DV[i][j] * Bc[3 * i + l] * T.DV[l][k] +
                         T.DX[i][j] * Cc[3 * i + l] * T.DV[l][k];
            F2[j][k] = s;
        }
    double e = f0 * m0;
    for (int j = 0; j < 3; ++j) {
        e += f1[j] * m1[j];
        for (int k = 0; k < 3; ++k) e += F2[j][k] * M2[j][k];
    }
    acc.I0 += T.mass * e;
    // dphi/dv = gv + G1 q, G1 = (B + B^T) DV + C^T DX;  J_k = mass E[lambda_k dphi/dv]
    double G1[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int l = 0; l < 3; ++l) s += (Bc[3 * i + l] + Bc[3 * l + i]) * T.DV[l][j] + Cc[3 * l + i] * T.DX[l][j];
            G1[i][j] = s;
        }
    double Jsum[3];
    for (int i = 0; i < 3; ++i) Jsum[i] = gv[i] * m0 + G1[i][0] * m1[0] + G1[i][1] * m1[1] + G1[i][2] * m1[2];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            const double t = gv[i] * m1[j] + G1[i][0] * M2[0][j] + G1[i][1] * M2[1][j] + G1[i][2] * M2[2][j];
            acc.J[j + 1][i] += T.mass * t;
            Jsum[i] -= t;
        }
    for (int i = 0; i < 3; ++i) acc.J[0][i] += T.mass * Jsum[i];
    // surface term: fan triangles of the faces that lie on a face of the tet
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
            // the face's tet-face tags: a face is on a tet face when all its vertices carry that tag
            uint32_t ft = tags(P.nb[vs]);
            {
                int wc = vs, wn = vn, st2 = 0;
                while (wn != vs) {
                    if (++st2 > WALK_CAP || wn >= P.nv) return ST_GRAPH;
                    const uint32_t w = P.nb[wn];
                    ft &= tags(w);
                    const int k = (nbget(w, 0) == wc) ? 0 : (nbget(w, 1) == wc) ? 1 : (nbget(w, 2) == wc) ? 2 : 3;
                    if (k == 3) return ST_GRAPH;
                    wc = wn;
                    wn = nbget(P.nb[wc], (k + 1) % 3);
                }
            }
            uint32_t w = P.nb[vn];
            int k = (nbget(w, 0) == vc) ? 0 : (nbget(w, 1) == vc) ? 1 : (nbget(w, 2) == vc) ? 2 : 3;
            if (k == 3) return ST_GRAPH;
            vc = vn;
            int kn = (k + 1) % 3;
            int b = 3 * vc + kn;
            done[b >> 6] |= 1ull << (b & 63);
            vn = nbget(P.nb[vc], kn);
            int steps = 0;
            while (vn != vs) {
                if (++steps > WALK_CAP || vn >= P.nv) return ST_GRAPH;
                if (ft) {
                    // triangle (vs, vn, vc) in the orientation of the q-space fan
                    const int tv[3] = {vs, vn, vc};
                    double e1[3], e2[3];
                    for (int i = 0; i < 3; ++i) {
                        e1[i] = (double)P.x[vn][i] - (double)P.x[vs][i];
                        e2[i] = (double)P.x[vc][i] - (double)P.x[vs][i];
                    }
                    const double N[3] = {0.5 * (e1[1] * e2[2] - e1[2] * e2[1]), 0.5 * (e1[2] * e2[0] - e1[0] * e2[2]),
                                         0.5 * (e1[0] * e2[1] - e1[1] * e2[0])};
                    double sl[4] = {0.0, 0.0, 0.0, 0.0};
                    // corners (1/20), edge midpoints (2/15), centroid (9/20)
                    for (int pnt = 0; pnt < 7; ++pnt) {
                        double wb[3], wt;
                        if (pnt < 3) {
                            wb[0] = wb[1] = wb[2] = 0.0;
                            wb[pnt] = 1.0;
                            wt = 1.0 / 20.0;
                        } else if (pnt < 6) {
                            wb[0] = wb[1] = wb[2] = 0.5;
                            wb[pnt - 3] = 0.0;
                            wt = 2.0 / 15.0;
                        } else {
                            wb[0] = wb[1] = wb[2] = 1.0 / 3.0;
                            wt = 9.0 / 20.0;
                        }
                        double q[3], x[3], v[3];
                        for (int i = 0; i < 3; ++i)
                            q[i] = wb[0] * (double)P.q[tv[0]][i] + wb[1] * (double)P.q[tv[1]][i] +
                                   wb[2] * (double)P.q[tv[2]][i];
                        for (int i = 0; i < 3; ++i) {
                            x[i] = T.x0[i] + T.DX[i][0] * q[0] + T.DX[i][1] * q[1] + T.DX[i][2] * q[2];
                            v[i] = T.v0[i] + T.DV[i][0] * q[0] + T.DV[i][1] * q[1] + T.DV[i][2] * q[2];
                        }
                        const double f = wt * phi(x, v);
                        sl[0] += f * (1.0 - q[0] - q[1] - q[2]);
                        sl[1] += f * q[0];
                        sl[2] += f * q[1];
                        sl[3] += f * q[2];
                    }
                    for (int kk = 0; kk < 4; ++kk)
                        for (int i = 0; i < 3; ++i) acc.bnd[kk][i] += sl[kk] * N[i];
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
