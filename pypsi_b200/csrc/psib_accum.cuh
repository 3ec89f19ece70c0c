// psib_accum.cuh -- physical moments of a central-form fragment, and their
// atomic accumulation into per-voxel sums (the fast, non-deterministic mode).
//
// A central-form fragment record is (m0, q-centroid cq, central q-space second
// moment C as xx xy xz yy yz zz).  Through the tet image's frame it becomes the
// fragment's mass, position and velocity centroids and its central second
// moments in x and v (src/geometry.c:81-161).  The per-voxel sums about the
// voxel's centre and its tile's reference velocity are merged into the grid
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

// Add fragment rec of image t, lying in voxel lo of grid g (global voxel gi,
// cutout `cut` of a batch, else 0), to the atomic sums, its mass scaled by
// `factor`.  x is taken about the voxel's centre, v about the tile's reference.
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
    double cm[3] = {0.0, 0.0, 0.0}, cv[3] = {0.0, 0.0, 0.0}, sxx[3][3], sxv[3][3], svv[3][3];
    mixed_fragment(rec, p0, DX, v0, DV, hx, hv, hxx, hxv, hvv, cm, cv, sxx, sxv, svv);
    double dx[3] = {0.0, 0.0, 0.0}, dv[3] = {0.0, 0.0, 0.0};
    if (hx)
        for (int i = 0; i < 3; ++i) {
            dx[i] = cm[i] - (g.w0[i] + g.d[i] * ((double)lo[i] + 0.5));
            atomicAdd(S + A.ox + i, m * dx[i]);
        }
    if (hv) {
        const long long tile = (A.toff ? A.toff[cut] : 0ll) + acc_tile(g, lo[0], lo[1], lo[2]);
        for (int i = 0; i < 3; ++i) {
            dv[i] = cv[i] - A.vref[3 * tile + i];
            atomicAdd(S + A.ov + i, m * dv[i]);
        }
    }
    int k = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j, ++k) {
            if (hxx) atomicAdd(S + A.oxx + k, m * (sxx[i][j] + dx[i] * dx[j]));
            if (hvv) atomicAdd(S + A.ovv + k, m * (svv[i][j] + dv[i] * dv[j]));
        }
    if (hxv)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) atomicAdd(S + A.oxv + 3 * i + j, m * (sxv[i][j] + dx[i] * dv[j]));
}

} // namespace psib
