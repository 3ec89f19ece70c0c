// tess.cu -- elements to tet images, and the per-voxel finalisation.
//
// Built with --fmad=false: the element unwrap, the trilinear refinement and
// the online field update below repeat the reference's double-precision
// operations in the reference's order.
#include <algorithm>

#include "psib_accum.cuh"
#include "psib_adjoint.cuh"
#include "psib_device.cuh"
#include "psib_kernels.h"

namespace psib {

// The 6-tet split of a 27-node cube, node indices 9i+3j+k (src/refine.c:39-41).
__constant__ int c_tet_nodes[6][4] = {{2, 0, 6, 18}, {8, 2, 6, 18}, {8, 20, 2, 18},
                                      {8, 24, 20, 18}, {8, 6, 24, 18}, {8, 26, 20, 24}};
// The same split on the 8 corner vertices 4i+2j+k of an unrefined element.
__constant__ int c_tet_corners[6][4] = {{1, 0, 2, 4}, {3, 1, 2, 4}, {3, 5, 1, 4},
                                        {3, 6, 5, 4}, {3, 2, 6, 4}, {3, 7, 5, 6}};
// Edges (end, midpoint, end) whose midpoint deviation drives refinement (src/refine.c:228-230).
__constant__ int c_ref_edges[7][3] = {{2, 4, 6}, {2, 10, 18}, {6, 12, 18}, {8, 13, 18},
                                      {8, 14, 20}, {8, 16, 24}, {20, 22, 24}};

// Edges (end, midpoint, end) of the tets of a 27-node cube whose midpoint deviation
// drives the refinement of a triquadratic element (src/refine.c:157-161).
__constant__ int c_quad_edges[19][3] = {{0, 1, 2},    {0, 3, 6},    {0, 9, 18},   {2, 4, 6},    {2, 5, 8},
                                        {2, 10, 18},  {2, 11, 20},  {6, 7, 8},    {6, 12, 18},  {6, 15, 24},
                                        {8, 13, 18},  {8, 14, 20},  {8, 16, 24},  {8, 17, 26},  {18, 19, 20},
                                        {18, 21, 24}, {20, 22, 24}, {20, 23, 26}, {24, 25, 26}};

constexpr int MAX_REFINE = 6; // src/refine.c:89-92

__device__ __forceinline__ int I2(int a, int b, int c) { return 4 * a + 2 * b + c; }
__device__ __forceinline__ int I3(int a, int b, int c) { return 9 * a + 3 * b + c; }

// 8 corners -> 27 nodes by repeated midpoints (src/refine.c:292-319).
__device__ void interp_trilinear(const double (*in)[3], double (*out)[3])
{
    for (int ax = 0; ax < 3; ++ax) {
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j)
                for (int k = 0; k < 2; ++k) out[I3(2 * i, 2 * j, 2 * k)][ax] = in[I2(i, j, k)][ax];
        for (int j = 0; j < 3; j += 2)
            for (int k = 0; k < 3; k += 2) out[I3(1, j, k)][ax] = 0.5 * (out[I3(0, j, k)][ax] + out[I3(2, j, k)][ax]);
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < 3; k += 2) out[I3(i, 1, k)][ax] = 0.5 * (out[I3(i, 0, k)][ax] + out[I3(i, 2, k)][ax]);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) out[I3(i, j, 1)][ax] = 0.5 * (out[I3(i, j, 0)][ax] + out[I3(i, j, 2)][ax]);
    }
}

// Gather an element's vertices; false if an id is out of range.
__device__ bool gather(const MeshDev& m, long long e, double (*p)[3], double (*u)[3], int* ids)
{
    const int et = m.elemtype;
    if (m.conn) {
        for (int v = 0; v < et; ++v) {
            const int id = m.conn[e * et + v];
            if (id < 0 || id >= m.npart) return false;
            ids[v] = id;
        }
    } else {
        // implicit block connectivity (src/PSI.c:644-656)
        const long long nyz = (long long)m.edim[1] * m.edim[2];
        const int i = (int)(e / nyz), j = (int)((e / m.edim[2]) % m.edim[1]), k = (int)(e % m.edim[2]);
        for (int ii = 0; ii < 2; ++ii)
            for (int jj = 0; jj < 2; ++jj)
                for (int kk = 0; kk < 2; ++kk)
                    ids[I2(ii, jj, kk)] = (int)((long long)m.bdim[1] * m.bdim[2] * ((i + ii) % m.bdim[0])
                                                + (long long)m.bdim[2] * ((j + jj) % m.bdim[1]) + ((k + kk) % m.bdim[2]));
    }
    for (int v = 0; v < et; ++v)
        for (int i = 0; i < 3; ++i) {
            p[v][i] = m.pos[3 * (long long)ids[v] + i];
            u[v][i] = m.vel ? m.vel[3 * (long long)ids[v] + i] : 0.0;
        }
    return true;
}

__device__ void aabb_n(const double (*p)[3], int n, double (*rb)[3])
{
    for (int i = 0; i < 3; ++i) {
        rb[0][i] = 1.0e30;
        rb[1][i] = -1.0e30;
    }
    for (int v = 0; v < n; ++v)
        for (int i = 0; i < 3; ++i) {
            if (p[v][i] < rb[0][i]) rb[0][i] = p[v][i];
            if (p[v][i] > rb[1][i]) rb[1][i] = p[v][i];
        }
}

// Unwrap an element that spans more than half the periodic box and cull it
// against the window (src/cpsi.c:309-341).
__device__ bool aabb_periodic(double (*p)[3], int n, const MeshDev& m, const GridDev& g)
{
    double rb[2][3];
    aabb_n(p, n, rb);
    if (m.periodic) {
        for (int i = 0; i < 3; ++i) {
            const double span = m.box1[i] - m.box0[i];
            if (rb[1][i] - rb[0][i] > 0.5 * span) {
                rb[0][i] = 1.0e30;
                rb[1][i] = -1.0e30;
                for (int v = 0; v < n; ++v) {
                    if (p[v][i] > m.box0[i] + 0.5 * span) p[v][i] -= span;
                    if (p[v][i] < rb[0][i]) rb[0][i] = p[v][i];
                    if (p[v][i] > rb[1][i]) rb[1][i] = p[v][i];
                }
            }
            if (rb[0][i] > g.w1[i]) return false;
            if (rb[1][i] < g.w0[i] && rb[0][i] + span > g.w1[i]) return false;
        }
    } else {
        for (int i = 0; i < 3; ++i) {
            if (rb[0][i] > g.w1[i]) return false;
            if (rb[1][i] < g.w0[i]) return false;
        }
    }
    return true;
}

// Periodic images of one tet (src/cpsi.c:343-373): image 0 is the tet itself,
// image s (bit i set = shifted by +span_i) exists when the tet reaches below
// box0 on every axis of s and the shifted box meets the window.  Images whose
// box lies outside the window are dropped here: the window clip would empty
// them (smax <= 0 at src/geometry.c:430).  Returns a mask of kept images.
__device__ unsigned tet_images(const double (*p)[3], const MeshDev& m, const GridDev& g, double (*rb)[3])
{
    aabb_n(p, 4, rb);
    unsigned flags = 0, keep = 0;
    if (m.periodic)
        for (int i = 0; i < 3; ++i)
            if (rb[0][i] < m.box0[i]) flags |= 1u << i;
    for (int s = 0; s < 8; ++s) {
        if ((flags & s) != (unsigned)s) continue;
        bool ok = true;
        for (int i = 0; i < 3; ++i) {
            const double sh = (m.box1[i] - m.box0[i]) * (1 & (s >> i));
            const double a = (s ? rb[0][i] + sh : rb[0][i]), b = (s ? rb[1][i] + sh : rb[1][i]);
            if (s && (a > g.w1[i] || b < g.w0[i])) ok = false;  // the reference's own image test
            if (b <= g.w0[i] || a >= g.w1[i]) ok = false;        // nothing inside the window
        }
        if (ok) keep |= 1u << s;
    }
    return keep;
}

// Ordering key of an image from its voxel index box (src/geometry.c:838-841):
// KEY_DEEP for images the deep-tree kernel takes -- bisection trees deeper
// than the main kernel serves (DMAX_MAIN), or boxes longer than SPAN_MAX voxels
// on an axis, where FP32 coordinates would lose too much precision inside a
// voxel -- otherwise larger boxes first, then by coarse cell (psib_kernels.h).
__device__ uint16_t footprint_key(const double (*rb)[3], const GridDev& g, const int* cbits)
{
    int depth = 0, span = 0, cell = 0;
    long long vol = 1;
    for (int i = 0; i < 3; ++i) {
        double cmin = rb[0][i], cmax = rb[1][i];
        if (g.w0[i] > cmin) cmin = g.w0[i];
        if (g.w1[i] < cmax) cmax = g.w1[i];
        int lo = (int)floor((cmin - g.w0[i]) / g.d[i]);
        int hi = (int)ceil((cmax - g.w0[i]) / g.d[i]);
        if (lo < 0) lo = 0;
        if (hi > g.n[i]) hi = g.n[i];
        const int sz = hi - lo;
        if (sz > 1) depth += 32 - __clz(sz - 1);
        if (sz > span) span = sz;
        if (vol < 0xFFFF) vol *= (sz > 1 ? sz : 1);
        const int ci = g.n[i] > 0 ? (int)(((long long)lo << cbits[i]) / g.n[i]) : 0;
        cell = (cell << cbits[i]) | (ci < (1 << cbits[i]) ? ci : (1 << cbits[i]) - 1);
    }
    if (depth > DMAX_MAIN || span > SPAN_MAX) return (uint16_t)KEY_DEEP;
    return (uint16_t)(((256 - vol) << KEY_CELL_BITS) | (cell << (KEY_CELL_BITS - cbits[0] - cbits[1] - cbits[2])));
}

struct Emitter {
    const TessArgs& a;
    const MeshDev& m; // the element's mesh and grid (its cutout's in a batch)
    const GridDev& g;
    int gid;          // the cutout
    bool write;      // false: count only
    long long pos;   // next item index (emit)
    int n;           // items so far
    unsigned long long tets;
    __device__ void tet(const double (*p)[3], const double (*u)[3], double mass, long long e, const int* pid)
    {
        double rb[2][3];
        const unsigned keep = tet_images(p, m, g, rb);
        tets++;
        for (int s = 0; s < 8; ++s) {
            if (!((keep >> s) & 1u)) continue;
            if (write) {
                const long long t = pos++;
                const long long cap = a.it.cap;
                if (t >= cap) { // a fixed-size item buffer (capture mode) that the images outgrew
                    atomicOr(a.status, ST_OVERFLOW);
                    n++;
                    continue;
                }
                double q[4][3], rq[2][3];
                double* fr = a.it.frame + t * FRAME;
                for (int v = 0; v < 4; ++v)
                    for (int i = 0; i < 3; ++i) {
                        const double sh = (m.box1[i] - m.box0[i]) * (1 & (s >> i));
                        q[v][i] = s ? p[v][i] + sh : p[v][i];
                        fr[3 * v + i] = q[v][i];
                        fr[FR_U + 3 * v + i] = u[v][i];
                    }
                for (int i = 0; i < 3; ++i) {
                    const double sh = (m.box1[i] - m.box0[i]) * (1 & (s >> i));
                    rq[0][i] = s ? rb[0][i] + sh : rb[0][i];
                    rq[1][i] = s ? rb[1][i] + sh : rb[1][i];
                }
                fr[FR_MASS] = mass;
                fr[FR_MASS + 1] = 0.0;
                a.it.elem[t] = (int)e;
                for (int v = 0; v < 4; ++v) a.it.pid[v * cap + t] = pid ? pid[v] : -1;
                a.it.key[t] = footprint_key(rq, g, a.cbits);
                if (a.it.grid) a.it.grid[t] = (uint16_t)gid;
            }
            n++;
        }
    }
};

struct RefNode {
    double p[27][3];
    double u[27][3];
    double mass;
    int child;
    int o[3], side; // the (sub)cube in the element's unit cube, in units of 1/128
};

// The pid entries of leaf tet t of (sub)cube N at level d: each vertex's place in the element.
__device__ __forceinline__ void leaf_codes(const RefNode& N, int t, int d, int* pc)
{
    const int h = N.side >> 1;
    for (int v = 0; v < 4; ++v) {
        const int nd = c_tet_nodes[t][v];
        pc[v] = refine_vertex_code(N.o[0] + (nd / 9) * h, N.o[1] + ((nd / 3) % 3) * h, N.o[2] + (nd % 3) * h, d);
    }
}

// The stretch criterion (PSIB_REFINE_STRETCH; the reference has only the
// midpoint test): refine a (sub)cube of level lvl whose edge along axis a is
// longer than T lag_a / 2^lvl, or whose volume (the sum of |volume| of its six
// tets) exceeds T lag_x lag_y lag_z / 8^lvl, lag being the Lagrangian cell.
// The oracle states the same test in the same operation order.
__device__ bool stretch_refine(const double (*p)[3], int lvl, double T, const double* lag)
{
    const double s = 1.0 / (double)(1 << lvl);
    for (int a = 0; a < 3; ++a) {
        const double lim = T * lag[a] * s;
        for (int u = 0; u < 3; u += 2)
            for (int w = 0; w < 3; w += 2) {
                const int i0 = a == 0 ? I3(0, u, w) : a == 1 ? I3(u, 0, w) : I3(u, w, 0);
                const int i1 = a == 0 ? I3(2, u, w) : a == 1 ? I3(u, 2, w) : I3(u, w, 2);
                double d2 = 0.0;
                for (int c = 0; c < 3; ++c) d2 += (p[i1][c] - p[i0][c]) * (p[i1][c] - p[i0][c]);
                if (d2 > lim * lim) return true;
            }
    }
    double vol = 0.0;
    for (int t = 0; t < 6; ++t) {
        const double* q0 = p[c_tet_nodes[t][0]];
        double e[3][3];
        for (int v = 0; v < 3; ++v)
            for (int c = 0; c < 3; ++c) e[v][c] = p[c_tet_nodes[t][v + 1]][c] - q0[c];
        const double det = e[0][0] * (e[1][1] * e[2][2] - e[1][2] * e[2][1]) -
                           e[0][1] * (e[1][0] * e[2][2] - e[1][2] * e[2][0]) +
                           e[0][2] * (e[1][0] * e[2][1] - e[1][1] * e[2][0]);
        vol += fabs(det);
    }
    return vol / 6.0 > T * lag[0] * lag[1] * lag[2] * (s * s * s);
}

// Adaptive refinement of a trilinear element, depth first in the reference's
// child order (src/refine.c:223-289).
template <class EM>
__device__ void refine_element(EM& em, const double (*cp)[3], const double (*cu)[3], double mass, long long e,
                               int max_lvl, double ptol2, int mode, double T, const double* lag, RefNode* L)
{
    interp_trilinear(cp, L[0].p);
    interp_trilinear(cu, L[0].u);
    L[0].mass = mass;
    L[0].child = -1;
    L[0].o[0] = L[0].o[1] = L[0].o[2] = 0;
    L[0].side = 128;
    int d = 0;
    while (d >= 0) {
        RefNode& N = L[d];
        if (N.child < 0) {
            bool refine = false;
            if (d < max_lvl && mode == 1) refine = stretch_refine(N.p, d, T, lag);
            else if (d < max_lvl)
                for (int k = 0; k < 7 && !refine; ++k) {
                    double err2 = 0.0;
                    for (int i = 0; i < 3; ++i) {
                        const double mt = 0.5 * (N.p[c_ref_edges[k][0]][i] + N.p[c_ref_edges[k][2]][i]);
                        const double ml = N.p[c_ref_edges[k][1]][i];
                        err2 += (mt - ml) * (mt - ml);
                    }
                    refine = err2 > ptol2;
                }
            if (!refine) {
                for (int t = 0; t < 6; ++t) {
                    double tp[4][3], tu[4][3];
                    for (int v = 0; v < 4; ++v)
                        for (int i = 0; i < 3; ++i) {
                            tp[v][i] = N.p[c_tet_nodes[t][v]][i];
                            tu[v][i] = N.u[c_tet_nodes[t][v]][i];
                        }
                    int pc[4];
                    leaf_codes(N, t, d, pc);
                    em.tet(tp, tu, N.mass * (1.0 / 6), e, pc);
                }
                d--;
                continue;
            }
            N.child = 0;
        }
        if (N.child < 8) {
            const int c = N.child++;
            const int ci = c >> 2, cj = (c >> 1) & 1, ck = c & 1;
            double kp[8][3], ku[8][3];
            for (int a = 0; a < 2; ++a)
                for (int b = 0; b < 2; ++b)
                    for (int cc = 0; cc < 2; ++cc)
                        for (int i = 0; i < 3; ++i) {
                            kp[I2(a, b, cc)][i] = N.p[I3(a + ci, b + cj, cc + ck)][i];
                            ku[I2(a, b, cc)][i] = N.u[I3(a + ci, b + cj, cc + ck)][i];
                        }
            interp_trilinear(kp, L[d + 1].p);
            interp_trilinear(ku, L[d + 1].u);
            L[d + 1].mass = 0.125 * N.mass;
            L[d + 1].child = -1;
            L[d + 1].side = N.side >> 1;
            L[d + 1].o[0] = N.o[0] + ci * L[d + 1].side;
            L[d + 1].o[1] = N.o[1] + cj * L[d + 1].side;
            L[d + 1].o[2] = N.o[2] + ck * L[d + 1].side;
            d++;
        } else {
            d--;
        }
    }
}

// Triquadratic interpolation of a 27-node cube onto the 125 nodes of its
// half-size lattice (src/refine.c:321-345), one node at a time: node (A,B,C)
// of the 5-lattice (A,B,C in 0..4).  The reference fills the lattice in three
// sweeps -- x on the even y,z planes, then y on the even z planes, then z --
// each new node 0.125 (3 n_near + 6 n_mid - n_far) of the three nodes before it
// on its line; these functions evaluate the same expressions on the same
// operands, so every node has the reference's value bit for bit.
__device__ __forceinline__ double quad_line(int a, double n0, double n2, double n4)
{
    return a == 1 ? 0.125 * (3.0 * n0 + 6.0 * n2 - n4) : 0.125 * (3.0 * n4 + 6.0 * n2 - n0);
}
__device__ double quad_x(const double (*in)[3], int A, int B, int C, int ax) // B, C even
{
    if (!(A & 1)) return in[I3(A >> 1, B >> 1, C >> 1)][ax];
    return quad_line(A, in[I3(0, B >> 1, C >> 1)][ax], in[I3(1, B >> 1, C >> 1)][ax], in[I3(2, B >> 1, C >> 1)][ax]);
}
__device__ double quad_y(const double (*in)[3], int A, int B, int C, int ax) // C even
{
    if (!(B & 1)) return quad_x(in, A, B, C, ax);
    return quad_line(B, quad_x(in, A, 0, C, ax), quad_x(in, A, 2, C, ax), quad_x(in, A, 4, C, ax));
}
__device__ double quad_node(const double (*in)[3], int A, int B, int C, int ax)
{
    if (!(C & 1)) return quad_y(in, A, B, C, ax);
    return quad_line(C, quad_y(in, A, B, 0, ax), quad_y(in, A, B, 2, ax), quad_y(in, A, B, 4, ax));
}

// Adaptive refinement of a triquadratic element, depth first in the reference's
// child order (src/refine.c:152-221): a cube is cut into 8 when the midpoint of
// one of its 19 tet edges deviates from the straight edge by more than the
// tolerance; child (i,j,k) takes nodes (2i..2i+2, ...) of the parent's
// 125-node interpolation; a leaf gives the 6 tets of its corner nodes
// (src/refine.c:299-319).
template <class EM>
__device__ void refine_element_quad(EM& em, const double (*cp)[3], const double (*cu)[3], double mass,
                                    long long e, int max_lvl, double ptol2, int mode, double T, const double* lag,
                                    RefNode* L)
{
    for (int n = 0; n < 27; ++n)
        for (int i = 0; i < 3; ++i) {
            L[0].p[n][i] = cp[n][i];
            L[0].u[n][i] = cu[n][i];
        }
    L[0].mass = mass;
    L[0].child = -1;
    L[0].o[0] = L[0].o[1] = L[0].o[2] = 0;
    L[0].side = 128;
    int d = 0;
    while (d >= 0) {
        RefNode& N = L[d];
        if (N.child < 0) {
            bool refine = false;
            if (d < max_lvl && mode == 1) refine = stretch_refine(N.p, d, T, lag);
            else if (d < max_lvl)
                for (int k = 0; k < 19 && !refine; ++k) {
                    double err2 = 0.0;
                    for (int i = 0; i < 3; ++i) {
                        const double mt = 0.5 * (N.p[c_quad_edges[k][0]][i] + N.p[c_quad_edges[k][2]][i]);
                        const double mq = N.p[c_quad_edges[k][1]][i];
                        err2 += (mt - mq) * (mt - mq);
                    }
                    refine = err2 > ptol2;
                }
            if (!refine) {
                for (int t = 0; t < 6; ++t) {
                    double tp[4][3], tu[4][3];
                    for (int v = 0; v < 4; ++v)
                        for (int i = 0; i < 3; ++i) {
                            tp[v][i] = N.p[c_tet_nodes[t][v]][i];
                            tu[v][i] = N.u[c_tet_nodes[t][v]][i];
                        }
                    int pc[4];
                    leaf_codes(N, t, d, pc);
                    em.tet(tp, tu, N.mass * (1.0 / 6), e, pc);
                }
                d--;
                continue;
            }
            N.child = 0;
        }
        if (N.child < 8) {
            const int c = N.child++;
            const int ci = c >> 2, cj = (c >> 1) & 1, ck = c & 1;
            RefNode& K = L[d + 1];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    for (int cc = 0; cc < 3; ++cc)
                        for (int i = 0; i < 3; ++i) {
                            K.p[I3(a, b, cc)][i] = quad_node(N.p, a + 2 * ci, b + 2 * cj, cc + 2 * ck, i);
                            K.u[I3(a, b, cc)][i] = quad_node(N.u, a + 2 * ci, b + 2 * cj, cc + 2 * ck, i);
                        }
            K.mass = 0.125 * N.mass;
            K.child = -1;
            K.side = N.side >> 1;
            K.o[0] = N.o[0] + ci * K.side;
            K.o[1] = N.o[1] + cj * K.side;
            K.o[2] = N.o[2] + ck * K.side;
            d++;
        } else {
            d--;
        }
    }
}

template <bool REFINE, bool QUAD>
__device__ int element_items(const TessArgs& a, const MeshDev& m, const GridDev& g, int gid, bool write, long long e,
                             long long pos, unsigned long long& tets, RefNode* L)
{
    constexpr int NV = QUAD ? 27 : 8; // vertices an element may have
    double p[NV][3], u[NV][3];
    int ids[NV];
    if (!QUAD && m.elemtype == 27) {
        atomicOr(a.status, ST_INDEX); // launched without the triquadratic variant
        return 0;
    }
    if (!gather(m, e, p, u, ids)) {
        atomicOr(a.status, ST_INDEX);
        return 0;
    }
    const int et = m.elemtype;
    if (!aabb_periodic(p, et, m, g)) return 0;
    const double me = m.mass ? m.mass[e] : 1.0;
    Emitter em{a, m, g, gid, write, pos, 0, 0};
    if (et == 4) {
        em.tet(p, u, me, e, ids); // a simplex element is one tet (src/refine.c:60-66)
    } else if (QUAD && et == 27) {
        if constexpr (QUAD)
            refine_element_quad(em, p, u, me, e, REFINE ? a.max_lvl : 0, m.ptol2, a.refine_mode, a.stretch, m.lag,
                                L);
    } else if (!REFINE) {
        for (int t = 0; t < 6; ++t) {
            double tp[4][3], tu[4][3];
            int pid[4];
            for (int v = 0; v < 4; ++v) {
                const int c = c_tet_corners[t][v];
                pid[v] = ids[c];
                for (int i = 0; i < 3; ++i) {
                    tp[v][i] = p[c][i];
                    tu[v][i] = u[c][i];
                }
            }
            em.tet(tp, tu, me * (1.0 / 6), e, pid);
        }
    } else {
        if constexpr (REFINE) refine_element(em, p, u, me, e, a.max_lvl, m.ptol2, a.refine_mode, a.stretch, m.lag, L);
    }
    tets += em.tets;
    return em.n;
}

template <bool REFINE, bool EMIT, bool QUAD>
__global__ void __launch_bounds__(128) k_tess(TessArgs a)
{
    RefNode* L = nullptr;
    RefNode Lbuf[(REFINE || QUAD) ? MAX_REFINE + 1 : 1];
    if constexpr (REFINE || QUAD) L = Lbuf;
    unsigned long long kept = 0, tets = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = a.e0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; e < a.e1; e += stride) {
        const long long pos = EMIT ? a.offset[e - a.e0] - a.offset_base : 0;
        int n;
        if (a.nbatch) {
            // the element's cutout: the last b with eoff[b] <= e
            int lo = 0, hi = a.nbatch;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (a.eoff[mid] <= e) lo = mid;
                else hi = mid;
            }
            n = element_items<REFINE, QUAD>(a, a.meshes[lo], a.grids[lo], lo, EMIT, e - a.eoff[lo], pos, tets, L);
        } else {
            n = element_items<REFINE, QUAD>(a, a.m, a.g, 0, EMIT, e, pos, tets, L);
        }
        if (!EMIT) a.count[e - a.e0] = n;
        kept += (n > 0);
    }
    if (a.counters && EMIT) {
        atomicAdd(&a.counters[0], kept);
        atomicAdd(&a.counters[1], tets);
    }
}

static int tess_grid(long long n)
{
    long long b = (n + 127) / 128;
    return (int)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

template <bool EMIT>
static void launch_tess(const TessArgs& a, cudaStream_t s)
{
    const int g = tess_grid(a.e1 - a.e0);
    const bool refine = a.max_lvl > 0 && (a.nbatch || a.m.elemtype != 4);
    if (a.quad) {
        if (refine) k_tess<true, EMIT, true><<<g, 128, 0, s>>>(a);
        else k_tess<false, EMIT, true><<<g, 128, 0, s>>>(a);
    } else {
        if (refine) k_tess<true, EMIT, false><<<g, 128, 0, s>>>(a);
        else k_tess<false, EMIT, false><<<g, 128, 0, s>>>(a);
    }
}

cudaError_t launch_tess_count(const TessArgs& a, cudaStream_t s)
{
    launch_tess<false>(a, s);
    return cudaGetLastError();
}

cudaError_t launch_tess_emit(const TessArgs& a, cudaStream_t s)
{
    launch_tess<true>(a, s);
    return cudaGetLastError();
}

// ---- annihilation: the tets of each element, from its unwrapped and its stored vertices ----

// Orientation and density of a tet as psi_orient_tet computes them
// (src/geometry.c:190-224): six times the signed volume is the triple product
// of the edges from vertex 3, a.x (b x c).x + b.x (c x a).x + c.x (a x b).x; a
// negative tet has vertices 0 and 1 swapped.  Orienting is idempotent (the
// swapped tet's volume is the exact negation), so orienting once here equals
// the reference's orienting at every use.  Writes a TREC record.
__device__ void ann_record(const double (*p)[3], double mass, double* r)
{
    double a[3], b[3], c[3];
    for (int i = 0; i < 3; ++i) {
        a[i] = p[0][i] - p[3][i];
        b[i] = p[1][i] - p[3][i];
        c[i] = p[2][i] - p[3][i];
    }
    const double s = a[0] * (b[1] * c[2] - b[2] * c[1]) + b[0] * (c[1] * a[2] - c[2] * a[1]) +
                     c[0] * (a[1] * b[2] - a[2] * b[1]);
    double vol = -(1.0 / 6.0) * s;
    const bool swap = vol < 0.0;
    if (swap) vol = -vol;
    for (int v = 0; v < 4; ++v) {
        const int src = swap && v < 2 ? 1 - v : v;
        for (int i = 0; i < 3; ++i) r[3 * v + i] = p[src][i];
    }
    r[TR_RHO] = mass / vol;
    r[TR_VOL] = vol;
    for (int i = 0; i < 3; ++i) {
        double lo = p[0][i], hi = p[0][i];
        for (int v = 1; v < 4; ++v) {
            lo = p[v][i] < lo ? p[v][i] : lo;
            hi = p[v][i] > hi ? p[v][i] : hi;
        }
        r[TR_BOX + i] = lo;
        r[TR_BOX + 3 + i] = hi;
    }
}

struct AnnEmitter {
    double* out; // null: count only
    long long pos;
    int n;
    unsigned long long tets;
    __device__ void tet(const double (*p)[3], const double (*)[3], double mass, long long, const int*)
    {
        if (out) ann_record(p, mass, out + (pos++) * TREC);
        n++;
        tets++;
    }
};

template <bool REFINE, bool QUAD>
__device__ int ann_side(const AnnTessArgs& a, const double (*p)[3], const double (*u)[3], double me, long long e,
                        double* out, long long pos, RefNode* L)
{
    AnnEmitter em{out, pos, 0, 0};
    const int et = a.m.elemtype;
    if (et == 4) {
        em.tet(p, u, me, e, nullptr);
    } else if (QUAD && et == 27) {
        if constexpr (QUAD) refine_element_quad(em, p, u, me, e, REFINE ? a.max_lvl : 0, a.m.ptol2, 0, 0.0, a.m.lag, L);
    } else if (!REFINE) {
        for (int t = 0; t < 6; ++t) {
            double tp[4][3];
            for (int v = 0; v < 4; ++v)
                for (int i = 0; i < 3; ++i) tp[v][i] = p[c_tet_corners[t][v]][i];
            em.tet(tp, tp, me * (1.0 / 6), e, nullptr);
        }
    } else {
        if constexpr (REFINE) refine_element(em, p, u, me, e, a.max_lvl, a.m.ptol2, 0, 0.0, a.m.lag, L);
    }
    return em.n;
}

// One thread per element: the cull of src/cpsi.c:88-93 (which unwraps the
// element), then its tets on side A (unwrapped vertices, the element loop of
// src/cpsi.c:95) and side B (stored vertices, the R*-tree partner of
// src/cpsi.c:123-131).  Count pass: tet counts and the unwrapped element box;
// emit pass: the tet records.
template <bool REFINE, bool QUAD, bool EMIT>
__global__ void __launch_bounds__(128) k_ann_tess(AnnTessArgs a)
{
    constexpr int NV = QUAD ? 27 : 8;
    RefNode* L = nullptr;
    RefNode Lbuf[(REFINE || QUAD) ? MAX_REFINE + 1 : 1];
    if constexpr (REFINE || QUAD) L = Lbuf;
    unsigned long long kept = 0, tets = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < a.m.nelem; e += stride) {
        double p[NV][3], u[NV][3], q[NV][3];
        int ids[NV];
        if ((!QUAD && a.m.elemtype == 27) || !gather(a.m, e, p, u, ids)) {
            atomicOr(a.status, ST_INDEX);
            if (!EMIT) a.cnt_a[e] = a.cnt_b[e] = 0;
            continue;
        }
        const int et = a.m.elemtype;
        for (int v = 0; v < et; ++v)
            for (int i = 0; i < 3; ++i) q[v][i] = p[v][i];
        const bool keep = aabb_periodic(q, et, a.m, a.g);
        if (!EMIT) {
            double rb[2][3];
            aabb_n(q, et, rb);
            for (int i = 0; i < 3; ++i) {
                a.ebox[6 * e + i] = rb[0][i];
                a.ebox[6 * e + 3 + i] = rb[1][i];
            }
        }
        if (!keep) {
            if (!EMIT) a.cnt_a[e] = a.cnt_b[e] = 0;
            continue;
        }
        const double me = a.m.mass ? a.m.mass[e] : 1.0;
        const int na = ann_side<REFINE, QUAD>(a, q, u, me, e, EMIT ? a.tets_a : nullptr, EMIT ? a.off_a[e] : 0, L);
        const int nb = ann_side<REFINE, QUAD>(a, p, u, me, e, EMIT ? a.tets_b : nullptr, EMIT ? a.off_b[e] : 0, L);
        if (!EMIT) {
            a.cnt_a[e] = na;
            a.cnt_b[e] = nb;
        }
        kept++;
        tets += na;
    }
    if (a.counters && EMIT) {
        atomicAdd(&a.counters[0], kept);
        atomicAdd(&a.counters[1], tets);
    }
}

cudaError_t launch_ann_tess(const AnnTessArgs& a, bool emit, cudaStream_t s)
{
    const int g = tess_grid(a.m.nelem);
    const bool refine = a.max_lvl > 0 && a.m.elemtype != 4;
    if (a.quad) {
        if (refine) emit ? k_ann_tess<true, true, true><<<g, 128, 0, s>>>(a) : k_ann_tess<true, true, false><<<g, 128, 0, s>>>(a);
        else emit ? k_ann_tess<false, true, true><<<g, 128, 0, s>>>(a) : k_ann_tess<false, true, false><<<g, 128, 0, s>>>(a);
    } else {
        if (refine) emit ? k_ann_tess<true, false, true><<<g, 128, 0, s>>>(a) : k_ann_tess<true, false, false><<<g, 128, 0, s>>>(a);
        else emit ? k_ann_tess<false, false, true><<<g, 128, 0, s>>>(a) : k_ann_tess<false, false, false><<<g, 128, 0, s>>>(a);
    }
    return cudaGetLastError();
}

// ---- element boxes and phase-space samples (queries, PSI.VDF) ----

// One thread per element: the cull against the window a.g (src/rtree.c:63-70,
// which unwraps the element) and its box; cnt_a[e] = cnt_b[e] = 1 when kept.
__global__ void __launch_bounds__(128) k_elem_boxes(AnnTessArgs a)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < a.m.nelem; e += stride) {
        double p[27][3], u[27][3];
        int ids[27];
        if (!gather(a.m, e, p, u, ids)) {
            atomicOr(a.status, ST_INDEX);
            a.cnt_a[e] = a.cnt_b[e] = 0;
            continue;
        }
        const bool keep = aabb_periodic(p, a.m.elemtype, a.m, a.g);
        double rb[2][3];
        aabb_n(p, a.m.elemtype, rb);
        for (int i = 0; i < 3; ++i) {
            a.ebox[6 * e + i] = rb[0][i];
            a.ebox[6 * e + 3 + i] = rb[1][i];
        }
        a.cnt_a[e] = a.cnt_b[e] = keep ? 1 : 0;
    }
}

cudaError_t launch_elem_boxes(const AnnTessArgs& a, cudaStream_t s)
{
    k_elem_boxes<<<tess_grid(a.m.nelem), 128, 0, s>>>(a);
    return cudaGetLastError();
}

// psi_barycentric (src/geometry.c:335-389): barycentric coordinates of s in
// the tet v, (w_i + s . n_i) / sum, where w_i is the volume term of the three
// vertices other than v[i] -- x_a (b x c).x + ... in the reference's order --
// and n_i the normal of the face opposite v[i], built from the same edge
// vectors as the reference's (those of its face planes); returns |sum| / 6.
__device__ __forceinline__ double cross_x(const double* a, const double* b) { return a[1] * b[2] - a[2] * b[1]; }

__device__ __forceinline__ void edge_cross(const double* a0, const double* a1, const double* b0, const double* b1,
                                           double* n)
{
    double A[3], B[3];
    for (int i = 0; i < 3; ++i) {
        A[i] = a1[i] - a0[i];
        B[i] = b1[i] - b0[i];
    }
    n[0] = A[1] * B[2] - A[2] * B[1];
    n[1] = A[2] * B[0] - A[0] * B[2];
    n[2] = A[0] * B[1] - A[1] * B[0];
}

__device__ double barycentric(const double (*v)[3], const double* s, double* b)
{
    double w[4], n[4][3];
    w[0] = v[1][0] * cross_x(v[2], v[3]) + v[2][0] * cross_x(v[3], v[1]) + v[3][0] * cross_x(v[1], v[2]);
    w[1] = v[0][0] * cross_x(v[3], v[2]) + v[2][0] * cross_x(v[0], v[3]) + v[3][0] * cross_x(v[2], v[0]);
    w[2] = v[0][0] * cross_x(v[1], v[3]) + v[1][0] * cross_x(v[3], v[0]) + v[3][0] * cross_x(v[0], v[1]);
    w[3] = v[0][0] * cross_x(v[2], v[1]) + v[1][0] * cross_x(v[0], v[2]) + v[2][0] * cross_x(v[1], v[0]);
    edge_cross(v[1], v[3], v[1], v[2], n[0]);
    edge_cross(v[0], v[2], v[2], v[3], n[1]);
    edge_cross(v[3], v[1], v[3], v[0], n[2]);
    edge_cross(v[2], v[0], v[0], v[1], n[3]);
    double tot = 0.0;
    for (int i = 0; i < 4; ++i) {
        b[i] = w[i];
        for (int j = 0; j < 3; ++j) b[i] += s[j] * n[i][j];
        tot += b[i];
    }
    for (int i = 0; i < 4; ++i) b[i] /= tot;
    return fabs((1.0 / 6.0) * tot);
}

// A tet that contains the point gives one sample: density mass / volume and
// the velocity interpolated at the point (src/cpsi.c:237-262).
struct VdfEmitter {
    const VdfArgs& a;
    const double* s;
    long long pos;   // next sample's index
    int n;
    bool write;
    long long cap;   // samples are written at indices below cap
    __device__ void tet(const double (*p)[3], const double (*u)[3], double mass, long long, const int*)
    {
        double b[4];
        const double vol = barycentric(p, s, b);
        if (vol <= 0.0) return;
        for (int i = 0; i < 4; ++i)
            if (b[i] < 0.0) return;
        if (write) {
            if (pos < cap) {
                for (int i = 0; i < 3; ++i) {
                    double acc = 0.0;
                    for (int j = 0; j < 4; ++j) acc += b[j] * u[j][i];
                    a.vel[3 * pos + i] = acc;
                }
                a.rho[pos] = mass / vol;
            }
            pos++;
        }
        n++;
    }
};

// The samples of one element at the emitter's point: the element refined from
// its vertices as stored (src/cpsi.c:222-230), every tet tested.
template <bool REFINE, bool QUAD>
__device__ void vdf_element(const VdfArgs& a, VdfEmitter& em, long long e, RefNode* L)
{
    constexpr int NV = QUAD ? 27 : 8;
    double p[NV][3], u[NV][3];
    int ids[NV];
    if ((!QUAD && a.m.elemtype == 27) || !gather(a.m, e, p, u, ids)) {
        atomicOr(a.status, ST_INDEX);
        return;
    }
    const double me = a.m.mass ? a.m.mass[e] : 1.0;
    const int et = a.m.elemtype;
    if (et == 4) {
        em.tet(p, u, me, e, nullptr);
    } else if (QUAD && et == 27) {
        if constexpr (QUAD)
            refine_element_quad(em, p, u, me, e, REFINE ? a.max_lvl : 0, a.m.ptol2, 0, 0.0, a.m.lag, L);
    } else if (!REFINE) {
        for (int t = 0; t < 6; ++t) {
            double tp[4][3], tu[4][3];
            for (int v = 0; v < 4; ++v)
                for (int c = 0; c < 3; ++c) {
                    tp[v][c] = p[c_tet_corners[t][v]][c];
                    tu[v][c] = u[c_tet_corners[t][v]][c];
                }
            em.tet(tp, tu, me * (1.0 / 6), e, nullptr);
        }
    } else {
        if constexpr (REFINE) refine_element(em, p, u, me, e, a.max_lvl, a.m.ptol2, 0, 0.0, a.m.lag, L);
    }
}

// One thread per (point, element) pair: the element refined from its vertices
// as stored (src/cpsi.c:222-230), every tet tested against the point.
template <bool REFINE, bool QUAD, bool EMIT>
__global__ void __launch_bounds__(128) k_vdf_samples(VdfArgs a)
{
    RefNode* L = nullptr;
    RefNode Lbuf[(REFINE || QUAD) ? MAX_REFINE + 1 : 1];
    if constexpr (REFINE || QUAD) L = Lbuf;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.npair; i += stride) {
        const unsigned long long key = a.pairs[i];
        const long long pt = (long long)(key >> 32);
        const long long e = (long long)(0xFFFFFFFFull - (key & 0xFFFFFFFFull));
        VdfEmitter em{a, a.points + 3 * pt, EMIT ? a.off[i] : 0, 0, EMIT, 0x7FFFFFFFFFFFFFFFll};
        vdf_element<REFINE, QUAD>(a, em, e, L);
        if (!EMIT) a.cnt[i] = em.n;
    }
}

// One point on one thread: its cell's elements in descending order (the pairs
// of k_query_points), each containing one sampled as above.
template <bool REFINE, bool QUAD>
__global__ void k_vdf_point(VdfArgs a, AnnArgs x, unsigned long long* count, long long cap)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    RefNode* L = nullptr;
    RefNode Lbuf[(REFINE || QUAD) ? MAX_REFINE + 1 : 1];
    if constexpr (REFINE || QUAD) L = Lbuf;
    const double* s = a.points;
    VdfEmitter em{a, s, 0, 0, true, cap};
    const long long r = find_run(x, point_cell(x.cg, s));
    if (r >= 0)
        for (long long j = x.run_off[r] + x.run_cnt[r] - 1; j >= x.run_off[r]; --j) {
            const long long e = x.reg_elem[j];
            bool in = true;
            for (int c = 0; c < 3; ++c)
                if (s[c] < x.ebox[6 * e + c] || s[c] > x.ebox[6 * e + 3 + c]) in = false;
            if (in) vdf_element<REFINE, QUAD>(a, em, e, L);
        }
    *count = (unsigned long long)em.n;
}

cudaError_t launch_vdf_point(const VdfArgs& a, const AnnArgs& x, unsigned long long* count, long long cap,
                             cudaStream_t s)
{
    const bool refine = a.max_lvl > 0 && a.m.elemtype != 4;
    if (a.quad) {
        if (refine) k_vdf_point<true, true><<<1, 32, 0, s>>>(a, x, count, cap);
        else k_vdf_point<false, true><<<1, 32, 0, s>>>(a, x, count, cap);
    } else {
        if (refine) k_vdf_point<true, false><<<1, 32, 0, s>>>(a, x, count, cap);
        else k_vdf_point<false, false><<<1, 32, 0, s>>>(a, x, count, cap);
    }
    return cudaGetLastError();
}

cudaError_t launch_vdf_samples(const VdfArgs& a, bool emit, cudaStream_t s)
{
    const int g = tess_grid(a.npair);
    const bool refine = a.max_lvl > 0 && a.m.elemtype != 4;
    if (a.quad) {
        if (refine) emit ? k_vdf_samples<true, true, true><<<g, 128, 0, s>>>(a) : k_vdf_samples<true, true, false><<<g, 128, 0, s>>>(a);
        else emit ? k_vdf_samples<false, true, true><<<g, 128, 0, s>>>(a) : k_vdf_samples<false, true, false><<<g, 128, 0, s>>>(a);
    } else {
        if (refine) emit ? k_vdf_samples<true, false, true><<<g, 128, 0, s>>>(a) : k_vdf_samples<true, false, false><<<g, 128, 0, s>>>(a);
        else emit ? k_vdf_samples<false, false, true><<<g, 128, 0, s>>>(a) : k_vdf_samples<false, false, false><<<g, 128, 0, s>>>(a);
    }
    return cudaGetLastError();
}

// ---- fragment records applied to the fields, voxel by voxel ----

// Sorted records into contiguous arrays: voxel, item, moments.
__global__ void k_gather_records(GatherArgs a)
{
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= a.nrec) return;
    const unsigned long long k = a.key[j];
    a.vox[j] = (unsigned)(k >> a.ibits);
    a.item[j] = (unsigned)(k & ((1ull << a.ibits) - 1ull));
    if (!a.mom_sorted) return; // central records are read through the permutation
    const double* src = a.mom + (long long)a.perm[j] * a.nmom;
    double* dst = a.mom_sorted + j * a.nmom;
    for (int m = 0; m < a.nmom; ++m) dst[m] = src[m];
}

cudaError_t launch_gather_records(const GatherArgs& a, cudaStream_t s)
{
    if (a.nrec == 0) return cudaSuccess;
    k_gather_records<<<(unsigned)((a.nrec + 255) / 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

// The fields of the run's voxel gv: its cutout's in a batch, with the voxel's
// index within that cutout.
struct Fields {
    double *M, *X, *V, *XX, *XV, *VV;
    long long gi;
};
__device__ __forceinline__ Fields fields_of(const ApplyArgs& a, long long gv)
{
    if (!a.nbatch) return Fields{a.M, a.X, a.V, a.XX, a.XV, a.VV, gv};
    int lo = 0, hi = a.nbatch;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (a.voff[mid] <= (unsigned long long)gv) lo = mid;
        else hi = mid;
    }
    double* const* f = a.fptr + 6 * lo;
    return Fields{f[0], f[1], f[2], f[3], f[4], f[5], gv - (long long)a.voff[lo]};
}

// One thread per voxel run walks the run in item order and applies
// src/geometry.c:106-186 exactly as the reference does.  For raw FP64 records
// this reproduces the reference's fields bit for bit.  The voxel's fields are
// held in registers for the whole run and stored once.
__global__ void __launch_bounds__(128) k_apply_runs(ApplyArgs a)
{
    const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= a.nruns) return;
    const Fields F = fields_of(a, (long long)a.run_vox[r]);
    const long long gi = F.gi;
    const long long beg = a.run_off[r], end = beg + a.run_cnt[r];
    const bool hx = a.X, hv = a.V, hxx = a.XX, hxv = a.XV, hvv = a.VV;
    double M = F.M[gi], X[3] = {0, 0, 0}, V[3] = {0, 0, 0}, XX[9], XV[9], VV[9];
    for (int i = 0; i < 3; ++i) {
        if (hx) X[i] = F.X[3 * gi + i];
        if (hv) V[i] = F.V[3 * gi + i];
    }
    for (int k = 0; k < 9; ++k) {
        XX[k] = hxx ? F.XX[9 * gi + k] : 0.0;
        XV[k] = hxv ? F.XV[9 * gi + k] : 0.0;
        VV[k] = hvv ? F.VV[9 * gi + k] : 0.0;
    }
    for (long long j = beg; j < end; ++j) {
        const long long t = a.item_base + (long long)a.item[j];
        const double* mom = a.mom + j * a.nmom;
        const double* fr = a.it.frame + t * FRAME;
        double p0[3], v0[3], DX[3][3], DV[3][3];
        for (int i = 0; i < 3; ++i) {
            p0[i] = fr[i];
            v0[i] = fr[FR_U + i];
            for (int k = 0; k < 3; ++k) {
                DX[i][k] = fr[3 * (k + 1) + i] - p0[i];
                DV[i][k] = fr[FR_U + 3 * (k + 1) + i] - v0[i];
            }
        }
        double mass = fr[FR_MASS];
        double cm[3], cv[3], sxx[3][3], sxv[3][3], svv[3][3];
        if (a.central) {
            mass *= a.scale[t];
            if (a.nmom > 1) mixed_fragment(mom, p0, DX, v0, DV, hx, hv, hxx, hxv, hvv, cm, cv, sxx, sxv, svv);
        } else {
            if (hx) centroid(mom, p0, DX, cm);
            if (hv) centroid(mom, v0, DV, cv);
            if (hxx) second_moment(mom, p0, cm, DX, p0, cm, DX, p0, cm, p0, cm, sxx);
            if (hxv) second_moment(mom, p0, cm, DX, v0, cv, DV, p0, cm, v0, cv, sxv);
            if (hvv) second_moment(mom, v0, cv, DV, v0, cv, DV, v0, cv, v0, cv, svv);
        }
        const double cw = mass * mom[0] / (M + mass * mom[0]);
        const double dw = M / (M + mass * mom[0]);
        if (hxx)
            for (int i = 0; i < 3; ++i)
                for (int j2 = 0; j2 < 3; ++j2)
                    XX[3 * i + j2] = dw * XX[3 * i + j2] + cw * sxx[i][j2] + cw * dw * (cm[i] - X[i]) * (cm[j2] - X[j2]);
        if (hxv)
            for (int i = 0; i < 3; ++i)
                for (int j2 = 0; j2 < 3; ++j2)
                    XV[3 * i + j2] = dw * XV[3 * i + j2] + cw * sxv[i][j2] + cw * dw * (cm[i] - X[i]) * (cv[j2] - V[j2]);
        if (hvv)
            for (int i = 0; i < 3; ++i)
                for (int j2 = 0; j2 < 3; ++j2)
                    VV[3 * i + j2] = dw * VV[3 * i + j2] + cw * svv[i][j2] + cw * dw * (cv[i] - V[i]) * (cv[j2] - V[j2]);
        if (hx)
            for (int i = 0; i < 3; ++i) X[i] += cw * (cm[i] - X[i]);
        if (hv)
            for (int i = 0; i < 3; ++i) V[i] += cw * (cv[i] - V[i]);
        M += mass * mom[0];
    }
    F.M[gi] = M;
    for (int i = 0; i < 3; ++i) {
        if (hx) F.X[3 * gi + i] = X[i];
        if (hv) F.V[3 * gi + i] = V[i];
    }
    for (int k = 0; k < 9; ++k) {
        if (hxx) F.XX[9 * gi + k] = XX[k];
        if (hxv) F.XV[9 * gi + k] = XV[k];
        if (hvv) F.VV[9 * gi + k] = VV[k];
    }
}

// Central-form records (mixed precision and FP64-central): the update order
// within a voxel is free, because the merge of src/geometry.c:164-186 is
// associative in exact arithmetic -- the result is
//   M = sum m_f,  X = sum m_f x_f / M,
//   XX = (sum m_f S_f + sum m_f (x_f - X)(x_f - X)^T) / M   (XV, VV alike).
// A group of AG lanes takes one voxel run: each lane projects every AG-th
// record (read through the sort permutation) and sums m, m dx, m dv and
// m (S + dx dy^T) about the centroid of the run's first record (no
// cancellation in FP64); the group adds its lanes' sums with shuffles, and its
// first lane merges them once into the voxel's fields.
constexpr int AG = 8;

__device__ __forceinline__ double group_sum(double v)
{
#pragma unroll
    for (int o = AG / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

__global__ void __launch_bounds__(128) k_apply_central(ApplyArgs a)
{
    const long long gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long r = gid / AG;
    const int l = (int)(gid % AG);
    // whole groups run the shuffles; a group past the last run does nothing else
    const bool run_ok = r < a.nruns;
    const bool hx = a.X, hv = a.V, hxx = a.XX, hxv = a.XV, hvv = a.VV;
    const long long beg = run_ok ? a.run_off[r] : 0, cnt = run_ok ? a.run_cnt[r] : 0;
    double rx[3] = {0, 0, 0}, rv[3] = {0, 0, 0}; // reference point: the first record's centroids
    double sm = 0.0, sx[3] = {0, 0, 0}, sv[3] = {0, 0, 0}, sxx[6] = {0, 0, 0, 0, 0, 0}, svv[6] = {0, 0, 0, 0, 0, 0};
    double sxv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    auto project = [&](long long j, double& m, double* cm, double* cv, double (*Sxx)[3], double (*Sxv)[3],
                       double (*Svv)[3]) {
        const long long jj = beg + j;
        const long long t = a.item_base + (long long)a.item[jj];
        const double* mom = a.mom + (long long)a.perm[jj] * a.nmom;
        const double* fr = a.it.frame + t * FRAME;
        double p0[3], v0[3], DX[3][3], DV[3][3];
        for (int i = 0; i < 3; ++i) {
            p0[i] = fr[i];
            v0[i] = fr[FR_U + i];
            for (int k = 0; k < 3; ++k) {
                DX[i][k] = fr[3 * (k + 1) + i] - p0[i];
                DV[i][k] = fr[FR_U + 3 * (k + 1) + i] - v0[i];
            }
        }
        m = fr[FR_MASS] * a.scale[t] * mom[0];
        if (a.nmom > 1) mixed_fragment(mom, p0, DX, v0, DV, hx, hv, hxx, hxv, hvv, cm, cv, Sxx, Sxv, Svv);
    };
    auto accumulate = [&](double m, const double* cm, const double* cv, const double (*Sxx)[3],
                          const double (*Sxv)[3], const double (*Svv)[3]) {
        double dx[3], dv[3];
        for (int i = 0; i < 3; ++i) {
            dx[i] = cm[i] - rx[i];
            dv[i] = cv[i] - rv[i];
        }
        sm += m;
        for (int i = 0; i < 3; ++i) {
            sx[i] += m * dx[i];
            sv[i] += m * dv[i];
        }
        int k = 0;
        for (int i = 0; i < 3; ++i)
            for (int j2 = i; j2 < 3; ++j2, ++k) {
                if (hxx) sxx[k] += m * (Sxx[i][j2] + dx[i] * dx[j2]);
                if (hvv) svv[k] += m * (Svv[i][j2] + dv[i] * dv[j2]);
            }
        if (hxv)
            for (int i = 0; i < 3; ++i)
                for (int j2 = 0; j2 < 3; ++j2) sxv[3 * i + j2] += m * (Sxv[i][j2] + dx[i] * dv[j2]);
    };
    {
        // the first record of each lane; lane 0's (always present in a run) is the reference point,
        // broadcast by every lane of the warp outside any divergent loop
        double m = 0.0, cm[3] = {0, 0, 0}, cv[3] = {0, 0, 0}, Sxx[3][3], Sxv[3][3], Svv[3][3];
        const bool has = l < cnt;
        if (has) project(l, m, cm, cv, Sxx, Sxv, Svv);
        const int src = (threadIdx.x & 31) & ~(AG - 1);
        for (int i = 0; i < 3; ++i) {
            rx[i] = __shfl_sync(0xFFFFFFFFu, cm[i], src);
            rv[i] = __shfl_sync(0xFFFFFFFFu, cv[i], src);
        }
        if (has) accumulate(m, cm, cv, Sxx, Sxv, Svv);
    }
    for (long long j = AG + l; j < cnt; j += AG) {
        double m = 0.0, cm[3] = {0, 0, 0}, cv[3] = {0, 0, 0}, Sxx[3][3], Sxv[3][3], Svv[3][3];
        project(j, m, cm, cv, Sxx, Sxv, Svv);
        accumulate(m, cm, cv, Sxx, Sxv, Svv);
    }
    sm = group_sum(sm);
    for (int i = 0; i < 3; ++i) {
        if (hx || hxx || hxv) sx[i] = group_sum(sx[i]);
        if (hv || hvv || hxv) sv[i] = group_sum(sv[i]);
    }
    for (int k = 0; k < 6; ++k) {
        if (hxx) sxx[k] = group_sum(sxx[k]);
        if (hvv) svv[k] = group_sum(svv[k]);
    }
    if (hxv)
        for (int k = 0; k < 9; ++k) sxv[k] = group_sum(sxv[k]);
    if (!run_ok || l != 0 || !(sm > 0.0)) return;
    // this voxel's new fragments as one: mass, means, central (co)variances
    const Fields F = fields_of(a, (long long)a.run_vox[r]);
    const long long gi = F.gi;
    double xr[3], vr[3], dxr[3], dvr[3];
    for (int i = 0; i < 3; ++i) {
        dxr[i] = sx[i] / sm;
        dvr[i] = sv[i] / sm;
        xr[i] = rx[i] + dxr[i];
        vr[i] = rv[i] + dvr[i];
    }
    const double M0 = F.M[gi], Mf = M0 + sm;
    const double cw = sm / Mf, dw = M0 / Mf;
    // merged with what the voxel holds (src/geometry.c:164-186 for one combined fragment)
    double X0[3] = {0, 0, 0}, V0[3] = {0, 0, 0};
    for (int i = 0; i < 3; ++i) {
        if (hx) X0[i] = F.X[3 * gi + i];
        if (hv) V0[i] = F.V[3 * gi + i];
    }
    if (hxx) {
        int k = 0;
        double C[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j2 = i; j2 < 3; ++j2, ++k) C[i][j2] = C[j2][i] = sxx[k] / sm - dxr[i] * dxr[j2];
        for (int i = 0; i < 3; ++i)
            for (int j2 = 0; j2 < 3; ++j2) {
                double* t = &F.XX[9 * gi + 3 * i + j2];
                *t = dw * *t + cw * C[i][j2] + cw * dw * (xr[i] - X0[i]) * (xr[j2] - X0[j2]);
            }
    }
    if (hvv) {
        int k = 0;
        double C[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j2 = i; j2 < 3; ++j2, ++k) C[i][j2] = C[j2][i] = svv[k] / sm - dvr[i] * dvr[j2];
        for (int i = 0; i < 3; ++i)
            for (int j2 = 0; j2 < 3; ++j2) {
                double* t = &F.VV[9 * gi + 3 * i + j2];
                *t = dw * *t + cw * C[i][j2] + cw * dw * (vr[i] - V0[i]) * (vr[j2] - V0[j2]);
            }
    }
    if (hxv)
        for (int i = 0; i < 3; ++i)
            for (int j2 = 0; j2 < 3; ++j2) {
                const double C = sxv[3 * i + j2] / sm - dxr[i] * dvr[j2];
                double* t = &F.XV[9 * gi + 3 * i + j2];
                *t = dw * *t + cw * C + cw * dw * (xr[i] - X0[i]) * (vr[j2] - V0[j2]);
            }
    if (hx)
        for (int i = 0; i < 3; ++i) F.X[3 * gi + i] = X0[i] + cw * (xr[i] - X0[i]);
    if (hv)
        for (int i = 0; i < 3; ++i) F.V[3 * gi + i] = V0[i] + cw * (vr[i] - V0[i]);
    F.M[gi] = Mf;
}

cudaError_t launch_apply_records(const ApplyArgs& a, cudaStream_t s)
{
    if (a.nruns == 0) return cudaSuccess;
    if (a.central) {
        const long long threads = a.nruns * AG;
        k_apply_central<<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(a);
    } else {
        k_apply_runs<<<(unsigned)((a.nruns + 127) / 128), 128, 0, s>>>(a);
    }
    return cudaGetLastError();
}

// ---- coefficients of the full adjoint (psib_adjoint.cuh) ----

// Per voxel: the first variation of L per unit mass at (x, v) as a quadratic
// about the voxel's means X, V:
//   c0 = gM - (<gXX, XX> + <gVV, VV> + <gXV, XV>) / M,  cx = gX / M,  cv = gV / M,
//   A = gXX / M,  B = gVV / M,  C = gXV / M;  then X and V.
__global__ void k_adj_coeffs(AdjCoefArgs a)
{
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < a.nvox;
         v += (long long)gridDim.x * blockDim.x) {
        double* c = a.coef + v * ADJ_NCOEF;
        const double M = a.F[0][v];
        if (!(M > 0.0)) {
            for (int k = 0; k < ADJ_NCOEF; ++k) c[k] = 0.0;
            continue;
        }
        const double iM = 1.0 / M;
        double c0 = a.G[0] ? a.G[0][v] : 0.0;
        const int off[6] = {0, 0, 0, 7, 25, 16}; // where A (xx), C (xv), B (vv) go
        for (int f = 3; f < 6; ++f) {
            double dot = 0.0;
            for (int k = 0; k < 9; ++k) {
                const double g = a.G[f] ? a.G[f][9 * v + k] : 0.0;
                if (a.G[f]) dot += g * a.F[f][9 * v + k];
                c[off[f] + k] = g * iM;
            }
            c0 -= dot * iM;
        }
        c[0] = c0;
        for (int i = 0; i < 3; ++i) {
            c[1 + i] = a.G[1] ? a.G[1][3 * v + i] * iM : 0.0;
            c[4 + i] = a.G[2] ? a.G[2][3 * v + i] * iM : 0.0;
            c[34 + i] = a.F[1] ? a.F[1][3 * v + i] : 0.0;
            c[37 + i] = a.F[2] ? a.F[2][3 * v + i] : 0.0;
        }
    }
}

cudaError_t launch_adj_coeffs(const AdjCoefArgs& a, cudaStream_t s)
{
    if (a.nvox <= 0) return cudaSuccess;
    const long long blocks = std::min<long long>((a.nvox + 255) / 256, 148ll * 32);
    k_adj_coeffs<<<(unsigned)blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// ---- the atomic accumulation: reference velocities, mass corrections, finalize ----

__device__ __forceinline__ int cutout_of(const ApplyArgs& a, long long gv)
{
    int lo = 0, hi = a.nbatch;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (a.voff[mid] <= (unsigned long long)gv) lo = mid;
        else hi = mid;
    }
    return lo;
}

// One thread per voxel: the voxel's sums (about its centre and its tile's
// reference velocity) as one fragment of mass sm, mean xr, vr and central
// (co)variances, merged once into what the voxel holds -- the update of
// src/geometry.c:164-186 for one combined fragment, as k_apply_central does.
__global__ void __launch_bounds__(128) k_acc_finalize(FinalArgs a)
{
    const AccArgs& A = a.acc;
    const bool hx = a.ap.X, hv = a.ap.V, hxx = a.ap.XX, hxv = a.ap.XV, hvv = a.ap.VV;
    for (long long gv = a.v0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; gv < a.v1;
         gv += (long long)gridDim.x * blockDim.x) {
        const double* S = A.sum + gv * A.stride;
        const double sm = S[0];
        if (!(sm > 0.0)) continue;
        const int cut = a.ap.nbatch ? cutout_of(a.ap, gv) : 0;
        const Fields F = fields_of(a.ap, gv);
        const long long gi = F.gi;
        const GridDev& g = a.grids ? a.grids[cut] : a.g;
        const long long nyz = (long long)g.n[1] * g.n[2];
        const int ix[3] = {(int)(gi / nyz), (int)((gi / g.n[2]) % g.n[1]), (int)(gi % g.n[2])};
        double xr[3], vr[3], dxr[3] = {0.0, 0.0, 0.0}, dvr[3] = {0.0, 0.0, 0.0};
        if (A.ox >= 0) {
            double cen[3], r[3];
            for (int i = 0; i < 3; ++i) cen[i] = g.w0[i] + g.d[i] * ((double)ix[i] + 0.5);
            unpack_xref(A.rx[gv], cen, g.d, r);
            for (int i = 0; i < 3; ++i) {
                dxr[i] = S[A.ox + i] / sm;
                xr[i] = r[i] + dxr[i];
            }
        }
        if (A.ov >= 0) {
            const long long tile = (A.toff ? A.toff[cut] : 0ll) + acc_tile(g, ix[0], ix[1], ix[2]);
            double r[3];
            unpack_vref(A.rv[gv], A.vref + 3 * tile, r);
            for (int i = 0; i < 3; ++i) {
                dvr[i] = S[A.ov + i] / sm;
                vr[i] = r[i] + dvr[i];
            }
        }
        const double M0 = F.M[gi], Mf = M0 + sm;
        const double cw = sm / Mf, dw = M0 / Mf;
        double X0[3] = {0, 0, 0}, V0[3] = {0, 0, 0};
        for (int i = 0; i < 3; ++i) {
            if (hx || hxx || hxv) X0[i] = hx ? F.X[3 * gi + i] : 0.0;
            if (hv || hvv || hxv) V0[i] = hv ? F.V[3 * gi + i] : 0.0;
        }
        if (hxx) {
            int k = 0;
            double C[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = i; j < 3; ++j, ++k) C[i][j] = C[j][i] = S[A.oxx + k] / sm - dxr[i] * dxr[j];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double* t = &F.XX[9 * gi + 3 * i + j];
                    *t = dw * *t + cw * C[i][j] + cw * dw * (xr[i] - X0[i]) * (xr[j] - X0[j]);
                }
        }
        if (hvv) {
            int k = 0;
            double C[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = i; j < 3; ++j, ++k) C[i][j] = C[j][i] = S[A.ovv + k] / sm - dvr[i] * dvr[j];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double* t = &F.VV[9 * gi + 3 * i + j];
                    *t = dw * *t + cw * C[i][j] + cw * dw * (vr[i] - V0[i]) * (vr[j] - V0[j]);
                }
        }
        if (hxv)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    const double C = S[A.oxv + 3 * i + j] / sm - dxr[i] * dvr[j];
                    double* t = &F.XV[9 * gi + 3 * i + j];
                    *t = dw * *t + cw * C + cw * dw * (xr[i] - X0[i]) * (vr[j] - V0[j]);
                }
        if (hx)
            for (int i = 0; i < 3; ++i) F.X[3 * gi + i] = X0[i] + cw * (xr[i] - X0[i]);
        if (hv)
            for (int i = 0; i < 3; ++i) F.V[3 * gi + i] = V0[i] + cw * (vr[i] - V0[i]);
        F.M[gi] = Mf;
    }
}

cudaError_t launch_acc_finalize(const FinalArgs& a, int num_sms, cudaStream_t s)
{
    if (a.v1 <= a.v0) return cudaSuccess;
    const long long blocks = std::min<long long>((a.v1 - a.v0 + 127) / 128, (long long)num_sms * 16);
    k_acc_finalize<<<(unsigned)blocks, 128, 0, s>>>(a);
    return cudaGetLastError();
}

// Mass and momentum of the images whose first vertex lies in each tile.
__global__ void k_vref_accum(ItemArrays it, long long n, GridDev g0, const GridDev* grids, const long long* toff,
                             double* tsum, const long long* n_dev)
{
    if (n_dev) n = min(n, *n_dev);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int cut = grids ? (int)it.grid[t] : 0;
        const GridDev& g = grids ? grids[cut] : g0;
        const double* fr = it.frame + t * FRAME;
        int ix[3];
        for (int a = 0; a < 3; ++a) {
            double f = floor((fr[a] - g.w0[a]) / g.d[a]);
            if (!(f >= 0.0)) f = 0.0;
            ix[a] = f < (double)g.n[a] ? (int)f : g.n[a] - 1;
        }
        const long long tile = (toff ? toff[cut] : 0ll) + acc_tile(g, ix[0], ix[1], ix[2]);
        const double m = fr[FR_MASS];
        atomicAdd(&tsum[4 * tile], m);
        for (int a = 0; a < 3; ++a)
            atomicAdd(&tsum[4 * tile + 1 + a],
                      m * 0.25 * (fr[FR_U + a] + fr[FR_U + 3 + a] + fr[FR_U + 6 + a] + fr[FR_U + 9 + a]));
    }
}

__global__ void k_vref_fix(const double* tsum, long long ntiles, double* vref)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < ntiles; k += (long long)gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a) vref[3 * k + a] = tsum[4 * k] > 0.0 ? tsum[4 * k + 1 + a] / tsum[4 * k] : 0.0;
}

cudaError_t launch_vref(const ItemArrays& it, long long nitems, const GridDev& g, const GridDev* grids,
                        const AccArgs& acc, double* tsum, long long ntiles, int num_sms, cudaStream_t s,
                        const long long* n_items)
{
    if (nitems > 0) k_vref_accum<<<num_sms * 8, 256, 0, s>>>(it, nitems, g, grids, acc.toff, tsum, n_items);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_vref_fix<<<num_sms * 4, 256, 0, s>>>(tsum, ntiles, (double*)acc.vref);
    return cudaGetLastError();
}

__global__ void k_correction_select(ItemArrays it, const double* scale, long long n, double tol, int* list,
                                    uint16_t* keys, double* factor, unsigned long long* count, const long long* n_dev)
{
    if (n_dev) n = min(n, *n_dev);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const double sc = scale[t];
        if (it.key[t] < KEY_DEEP && sc > 0.0 && fabs(sc - 1.0) > tol) { // breadth-first images only
            const unsigned long long i = atomicAdd(count, 1ull);
            list[i] = (int)t;
            keys[i] = it.key[t];
            factor[t] = sc - 1.0;
        }
    }
}

cudaError_t launch_correction_select(const ItemArrays& it, const double* scale, long long nitems, double tol,
                                     int* list, uint16_t* keys, double* factor, unsigned long long* n, int num_sms,
                                     cudaStream_t s, const long long* n_items)
{
    if (nitems <= 0) return cudaSuccess;
    k_correction_select<<<num_sms * 8, 256, 0, s>>>(it, scale, nitems, tol, list, keys, factor, n, n_items);
    return cudaGetLastError();
}

} // namespace psib
