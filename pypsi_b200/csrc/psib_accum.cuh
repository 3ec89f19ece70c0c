// psib_accum.cuh -- physical moments of a central-form fragment, and their
// atomic accumulation into per-voxel sums (the fast, non-deterministic mode).
//
// A central-form fragment record is (m0, q-centroid cq, central q-space second
// moment C as xx xy xz yy yz zz).  Through the tet image's frame it becomes the
// fragment's mass, position and velocity centroids and its central second
// moments in x and v (src/geometry.c:81-161).  The per-voxel sums about the
// voxel's reference points (claimed by its first fragment) are merged into the grid
// fields by the finalize kernel (tess.cu), as the reference's online update
// (src/geometry.c:164-186) merges one combined fragment.
#pragma once
#include "psib_device.cuh"
#include "psib_kernels.h"

namespace psib {

// Physical moments of one central-form fragment: centroid c = x0 + D cq,
// central moment D C D^T.  The x-v moment is brought to the reference's
// pairing of its cross terms (src/geometry.c:137-146), which equals
// cov_xv + 2 a b^T - a a^T - b b^T with a = x0 - c_x and b = v0 - c_v.
__device__ __forceinline__ void mixed_fragment(const double* rec, const double* p0, const double (*DX)[3],
                                               const double* v0, const double (*DV)[3], bool x, bool v, bool xx,
                                               bool xv, bool vv, double* cm, double* cv, double (*sxx)[3],
                                               double (*sxv)[3], double (*svv)[3])
{
    const double* cq = rec + 1;
    // second moments are only recorded (and only read) when a second-order field is asked for
    const bool two = xx || xv || vv;
    const double C[3][3] = {{two ? rec[4] : 0.0, two ? rec[5] : 0.0, two ? rec[6] : 0.0},
                            {two ? rec[5] : 0.0, two ? rec[7] : 0.0, two ? rec[8] : 0.0},
                            {two ? rec[6] : 0.0, two ? rec[8] : 0.0, two ? rec[9] : 0.0}};
    if (x || xx || xv)
        for (int i = 0; i < 3; ++i) cm[i] = p0[i] + DX[i][0] * cq[0] + DX[i][1] * cq[1] + DX[i][2] * cq[2];
    if (v || xv || vv)
        for (int i = 0; i < 3; ++i) cv[i] = v0[i] + DV[i][0] * cq[0] + DV[i][1] * cq[1] + DV[i][2] * cq[2];
    double TX[3][3], TV[3][3];
    for (int i = 0; i < 3; ++i)
        for (int q = 0; q < 3; ++q) {
            TX[i][q] = (xx || xv) ? DX[i][0] * C[0][q] + DX[i][1] * C[1][q] + DX[i][2] * C[2][q] : 0.0;
            TV[i][q] = vv ? DV[i][0] * C[0][q] + DV[i][1] * C[1][q] + DV[i][2] * C[2][q] : 0.0;
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            if (xx) sxx[i][j] = TX[i][0] * DX[j][0] + TX[i][1] * DX[j][1] + TX[i][2] * DX[j][2];
            if (vv) svv[i][j] = TV[i][0] * DV[j][0] + TV[i][1] * DV[j][1] + TV[i][2] * DV[j][2];
            if (xv) {
                const double ai = p0[i] - cm[i], aj = p0[j] - cm[j], bi = v0[i] - cv[i], bj = v0[j] - cv[j];
                sxv[i][j] = TX[i][0] * DV[j][0] + TX[i][1] * DV[j][1] + TX[i][2] * DV[j][2] + 2.0 * ai * bj - ai * aj -
                            bi * bj;
            }
        }
}

// Reference points of a voxel, claimed by its first fragment.  A reference
// need not be exact, only near the voxel's means, and the same for every
// fragment of the voxel and for the finalize pass; so it is packed into one
// 64-bit word (top bit set: claimed) that a single atomicCAS publishes:
//   position: 3 x 21-bit fixed point, the offset from the voxel's centre in
//             units of d / 2^19 (the centroid lies within half a voxel);
//   velocity: 3 x 21-bit truncated floats (sign, exponent, 12 mantissa bits) of
//             the offset from the tile's reference velocity.
constexpr unsigned long long REF_SET = 1ull << 63;
constexpr double REF_QX = 524288.0; // 2^19 steps per voxel

__device__ __forceinline__ unsigned long long pack_xref(const double* c, const double* cen, const double* d)
{
    unsigned long long w = REF_SET;
    for (int i = 0; i < 3; ++i) {
        double q = rint((c[i] - cen[i]) / d[i] * REF_QX);
        q = fmin(fmax(q, -1048575.0), 1048575.0);
        w |= (unsigned long long)((long long)q + 1048576) << (42 - 21 * i);
    }
    return w;
}
__device__ __forceinline__ void unpack_xref(unsigned long long w, const double* cen, const double* d, double* r)
{
    for (int i = 0; i < 3; ++i)
        r[i] = cen[i] + (double)((long long)((w >> (42 - 21 * i)) & 0x1FFFFFull) - 1048576) * (d[i] / REF_QX);
}
__device__ __forceinline__ unsigned long long pack_vref(const double* off)
{
    unsigned long long w = REF_SET;
    for (int i = 0; i < 3; ++i) {
        const float f = isfinite(off[i]) ? (float)off[i] : 0.0f;
        w |= (unsigned long long)(__float_as_uint(f) >> 11) << (42 - 21 * i);
    }
    return w;
}
__device__ __forceinline__ void unpack_vref(unsigned long long w, const double* u, double* r)
{
    for (int i = 0; i < 3; ++i)
        r[i] = u[i] + (double)__uint_as_float((unsigned)((w >> (42 - 21 * i)) & 0x1FFFFFull) << 11);
}
// The word at *slot, claimed with `mine` if it is still 0.
__device__ __forceinline__ unsigned long long claim_ref(unsigned long long* slot, unsigned long long mine)
{
    const unsigned long long w = *(volatile unsigned long long*)slot;
    if (w) return w;
    const unsigned long long old = atomicCAS(slot, 0ull, mine);
    return old ? old : mine;
}

// Add fragment rec of image t, lying in voxel lo of grid g (global voxel gi,
// cutout `cut` of a batch, else 0), to the atomic sums, its mass scaled by
// `factor`.  x and v are taken about the voxel's reference points.
// Inlined into the leaf and clip kernels, whose register budgets are capped by
// their launch bounds.
__device__ __forceinline__ void accumulate_fragment(const ClipArgs& a, const GridDev& g, int cut, long long gi,
                                                    const int* lo, long long t, const double* rec, double factor)
{
    const AccArgs& A = a.acc;
    const double* fr = a.it.frame + t * FRAME;
    const bool hx = A.ox >= 0, hv = A.ov >= 0, hxx = A.oxx >= 0, hxv = A.oxv >= 0, hvv = A.ovv >= 0;
    double* S = A.sum + gi * A.stride;
    const double m = fr[FR_MASS] * factor * rec[0];
    atomicAdd(S, m);
    if (!(hx || hv)) return;
    double p0[3], v0[3], DX[3][3], DV[3][3];
    for (int i = 0; i < 3; ++i) {
        p0[i] = fr[i];
        v0[i] = fr[FR_U + i];
        for (int k = 0; k < 3; ++k) {
            DX[i][k] = fr[3 * (k + 1) + i] - p0[i];
            DV[i][k] = fr[FR_U + 3 * (k + 1) + i] - v0[i];
        }
    }
    // the projection of mixed_fragment, computed where its terms are added so that the matrices
    // of one field are dead before the next field's are formed (a smaller register peak in the
    // leaf and clip kernels that inline this)
    const double* cq = rec + 1;
    double cm[3] = {0.0, 0.0, 0.0}, cv[3] = {0.0, 0.0, 0.0};
    if (hx)
        for (int i = 0; i < 3; ++i) cm[i] = p0[i] + DX[i][0] * cq[0] + DX[i][1] * cq[1] + DX[i][2] * cq[2];
    if (hv)
        for (int i = 0; i < 3; ++i) cv[i] = v0[i] + DV[i][0] * cq[0] + DV[i][1] * cq[1] + DV[i][2] * cq[2];
    double dx[3] = {0.0, 0.0, 0.0}, dv[3] = {0.0, 0.0, 0.0};
    if (hx) {
        double cen[3], r[3];
        for (int i = 0; i < 3; ++i) cen[i] = g.w0[i] + g.d[i] * ((double)lo[i] + 0.5);
        unpack_xref(claim_ref(A.rx + gi, pack_xref(cm, cen, g.d)), cen, g.d, r);
        for (int i = 0; i < 3; ++i) {
            dx[i] = cm[i] - r[i];
            atomicAdd(S + A.ox + i, m * dx[i]);
        }
    }
    if (hv) {
        const long long tile = (A.toff ? A.toff[cut] : 0ll) + acc_tile(g, lo[0], lo[1], lo[2]);
        const double* u = A.vref + 3 * tile;
        const double off[3] = {cv[0] - u[0], cv[1] - u[1], cv[2] - u[2]};
        double r[3];
        unpack_vref(claim_ref(A.rv + gi, pack_vref(off)), u, r);
        for (int i = 0; i < 3; ++i) {
            dv[i] = cv[i] - r[i];
            atomicAdd(S + A.ov + i, m * dv[i]);
        }
    }
    if (!(hxx || hxv || hvv)) return;
    // central q-space second moment C of the fragment
    const double C[3][3] = {{rec[4], rec[5], rec[6]}, {rec[5], rec[7], rec[8]}, {rec[6], rec[8], rec[9]}};
    if (hxx || hxv) {
        double TX[3][3]; // DX C
        for (int i = 0; i < 3; ++i)
            for (int q = 0; q < 3; ++q) TX[i][q] = DX[i][0] * C[0][q] + DX[i][1] * C[1][q] + DX[i][2] * C[2][q];
        if (hxx) {
            int k = 0;
            for (int i = 0; i < 3; ++i)
                for (int j = i; j < 3; ++j, ++k) {
                    const double sxx = TX[i][0] * DX[j][0] + TX[i][1] * DX[j][1] + TX[i][2] * DX[j][2];
                    atomicAdd(S + A.oxx + k, m * (sxx + dx[i] * dx[j]));
                }
        }
        if (hxv)
            // the reference's pairing of the x-v cross terms (src/geometry.c:137-146):
            // cov_xv + 2 a b^T - a a^T - b b^T with a = x0 - c_x, b = v0 - c_v
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    const double ai = p0[i] - cm[i], aj = p0[j] - cm[j], bi = v0[i] - cv[i], bj = v0[j] - cv[j];
                    const double sxv = TX[i][0] * DV[j][0] + TX[i][1] * DV[j][1] + TX[i][2] * DV[j][2] +
                                       2.0 * ai * bj - ai * aj - bi * bj;
                    atomicAdd(S + A.oxv + 3 * i + j, m * (sxv + dx[i] * dv[j]));
                }
    }
    if (hvv) {
        double TV[3][3]; // DV C
        for (int i = 0; i < 3; ++i)
            for (int q = 0; q < 3; ++q) TV[i][q] = DV[i][0] * C[0][q] + DV[i][1] * C[1][q] + DV[i][2] * C[2][q];
        int k = 0;
        for (int i = 0; i < 3; ++i)
            for (int j = i; j < 3; ++j, ++k) {
                const double svv = TV[i][0] * DV[j][0] + TV[i][1] * DV[j][1] + TV[i][2] * DV[j][2];
                atomicAdd(S + A.ovv + k, m * (svv + dv[i] * dv[j]));
            }
    }
}

} // namespace psib
