/*
 * psi_oracle.c -- CPU restatement of PSI.voxels(grid, mesh) in density and
 * annihilation mode.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it; the
 * product library (pypsi_b200) never links, imports or calls anything here.
 *
 * It restates the reference algorithm of devonmpowell/PyPSI (files cited as
 * path:line inside that project) one step at a time, keeping every
 * floating-point operation in the reference's order so that, compiled with
 * -ffp-contract=off and no FMA, it reproduces the reference bit for bit.  That
 * claim is pinned by tests/test_oracle_pin.py against the reference's own
 * sources compiled into oracle/_ref/ (oracle/Makefile).
 *
 * Beyond the reference it keeps work counters (tets, tet images, fragments,
 * splits, fragment vertices) which give the algorithmic work units of a run.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Arithmetic type of the clip, moments and projection.  double (default)
 * repeats the reference bit for bit; building with -DOV_REAL=__float128 gives
 * an "exact" oracle (113-bit mantissa) that measures the reference's own
 * rounding error, which is large for tiny fragments: their raw q-moments about
 * the tet's vertex 0 cancel. */
#ifndef OV_REAL
#define OV_REAL double
#endif
typedef OV_REAL ov_real;

#define OV_MAXV 64        /* vertex buffer of one polyhedron (include/geometry.h:23) */
#define OV_STACK 64       /* bisection stack depth (src/geometry.c:41-46) */
#define OV_WALK_CAP 4096  /* bound on a face walk; the reference has none */

/* ---- public structs (mirrored by oracle/oracle.py with ctypes) ---- */

typedef struct {
    int n[3];
    double win[2][3];
    double d[3];
    double *f[6]; /* m, x, v, xx, xv, vv (include/grid.h:37-42); NULL when absent */
} og_grid;

typedef struct {
    int elemtype;            /* 4, 8 or 27 */
    int npart, nelem;
    const double *pos, *vel; /* npart x 3 */
    const double *mass;      /* nelem */
    const int *conn;         /* nelem x elemtype */
    int periodic;
    double box[2][3];
} og_mesh;

typedef struct {
    long long elements_kept; /* elements that survive the window cull */
    long long tets;          /* tets after refinement, without periodic images */
    long long tet_images;    /* tets including periodic images */
    long long fragments;     /* (tet image, voxel) pieces with m0 > 0 */
    long long splits;        /* calls of the axis-aligned split */
    long long frag_verts;    /* sum of vertex counts over emitted fragments */
    long long max_verts;     /* largest vertex count of any polyhedron seen */
    long long errors;        /* vertex-buffer overflow or a face walk that did not close */
} og_counters;

/* ---- polyhedron: r3d vertex graph with barycentric mass coordinates q ---- */

typedef struct {
    ov_real pos[3];
    ov_real q[3];
    int nbr[3];
} ov_vert;

typedef struct {
    int nv;
    int lo[3], hi[3]; /* voxel index box (src/geometry.c:838-841) */
    ov_vert v[OV_MAXV];
} ov_poly;

static og_counters *g_cnt;

static void note_nv(int nv)
{
    if (nv > g_cnt->max_verts) g_cnt->max_verts = nv;
}

/* Link each vertex created by a cut to its two neighbours on the cut face by
 * walking around the face it opens (src/geometry.c:459-482, :646-669). */
static int link_new_vertices(ov_poly *P, int onv, int nv)
{
    for (int vs = onv; vs < nv; ++vs) {
        int vc = vs, vn = P->v[vs].nbr[0], k = 0, steps = 0;
        do {
            for (k = 0; k < 3; ++k)
                if (P->v[vn].nbr[k] == vc) break;
            if (k == 3 || ++steps > OV_WALK_CAP) return -1;
            vc = vn;
            vn = P->v[vc].nbr[(k + 1) % 3];
        } while (vc < onv);
        P->v[vs].nbr[2] = vc;
        P->v[vc].nbr[1] = vs;
    }
    return 0;
}

/* Clip by half-spaces n.x + d >= 0 (src/geometry.c:391-501). */
static void ov_clip(ov_poly *P, const ov_real (*pn)[3], const ov_real *pd, int nplanes)
{
    if (P->nv <= 0) return;
    for (int p = 0; p < nplanes; ++p) {
        int onv = P->nv;
        ov_real s[OV_MAXV];
        int map[OV_MAXV];
        ov_real smin = 1.0e30, smax = -1.0e30;
        memset(map, 0, sizeof(map));
        for (int v = 0; v < onv; ++v) {
            s[v] = pd[p];
            for (int i = 0; i < 3; ++i) s[v] += P->v[v].pos[i] * pn[p][i];
            if (s[v] < smin) smin = s[v];
            if (s[v] > smax) smax = s[v];
            if (s[v] < 0.0) map[v] = 1;
        }
        if (smin >= 0.0) continue;
        if (smax <= 0.0) {
            P->nv = 0;
            return;
        }
        int nv = onv;
        for (int vc = 0; vc < onv; ++vc) {
            if (map[vc]) continue;
            for (int k = 0; k < 3; ++k) {
                int vn = P->v[vc].nbr[k];
                if (!map[vn]) continue;
                if (nv >= OV_MAXV) { g_cnt->errors++; P->nv = 0; return; }
                ov_real w = 1.0 / (s[vc] - s[vn]);
                ov_vert *a = &P->v[vc], *b = &P->v[vn], *c = &P->v[nv];
                for (int i = 0; i < 3; ++i) c->pos[i] = w * (b->pos[i] * s[vc] - a->pos[i] * s[vn]);
                for (int i = 0; i < 3; ++i) c->q[i] = w * (b->q[i] * s[vc] - a->q[i] * s[vn]);
                c->nbr[0] = vc;
                a->nbr[k] = nv;
                nv++;
            }
        }
        if (link_new_vertices(P, onv, nv)) { g_cnt->errors++; P->nv = 0; return; }
        note_nv(nv);
        int cnt = 0;
        for (int v = 0; v < nv; ++v) {
            if (!map[v]) {
                P->v[cnt] = P->v[v];
                map[v] = cnt++;
            }
        }
        P->nv = cnt;
        for (int v = 0; v < cnt; ++v)
            for (int k = 0; k < 3; ++k) P->v[v].nbr[k] = map[P->v[v].nbr[k]];
    }
}

/* Split by the plane x[ax] = coord into out[0] (x <= coord) and out[1]
 * (src/geometry.c:560-690).  `in` is used as scratch. */
static void ov_split(ov_poly *in, ov_poly *out, double coord, int ax)
{
    ov_real s[OV_MAXV];
    int side[OV_MAXV];
    int nright = 0, onv = in->nv;
    memset(side, 0, sizeof(side));
    g_cnt->splits++;
    for (int v = 0; v < onv; ++v) {
        s[v] = coord - in->v[v].pos[ax];
        if (s[v] < 0.0) {
            side[v] = 1;
            nright++;
        }
    }
    if (nright == 0) {
        out[0] = *in;
        out[1].nv = 0;
        return;
    }
    if (nright == onv) {
        out[1] = *in;
        out[0].nv = 0;
        return;
    }
    int nv = onv;
    for (int vc = 0; vc < onv; ++vc) {
        if (side[vc]) continue;
        for (int k = 0; k < 3; ++k) {
            int vn = in->v[vc].nbr[k];
            if (!side[vn]) continue;
            if (nv + 2 > OV_MAXV) { g_cnt->errors++; out[0].nv = out[1].nv = 0; return; }
            ov_real w = 1.0 / (s[vc] - s[vn]);
            ov_vert *a = &in->v[vc], *b = &in->v[vn];
            ov_real np_[3], nq[3];
            for (int i = 0; i < 3; ++i) {
                np_[i] = w * (b->pos[i] * s[vc] - a->pos[i] * s[vn]);
                nq[i] = w * (b->q[i] * s[vc] - a->q[i] * s[vn]);
            }
            ov_vert *l = &in->v[nv], *r = &in->v[nv + 1];
            memcpy(l->pos, np_, sizeof(np_));
            memcpy(l->q, nq, sizeof(nq));
            l->nbr[0] = vc;
            a->nbr[k] = nv;
            memcpy(r->pos, np_, sizeof(np_));
            memcpy(r->q, nq, sizeof(nq));
            side[nv + 1] = 1;
            r->nbr[0] = vn;
            int kb;
            for (kb = 0; kb < 3; ++kb)
                if (b->nbr[kb] == vc) break;
            if (kb == 3) { g_cnt->errors++; out[0].nv = out[1].nv = 0; return; }
            b->nbr[kb] = nv + 1;
            nv += 2;
        }
    }
    if (link_new_vertices(in, onv, nv)) { g_cnt->errors++; out[0].nv = out[1].nv = 0; return; }
    note_nv(nv);
    out[0].nv = 0;
    out[1].nv = 0;
    for (int v = 0; v < nv; ++v) {
        ov_poly *o = &out[side[v]];
        o->v[o->nv] = in->v[v];
        side[v] = o->nv++;
    }
    for (int h = 0; h < 2; ++h)
        for (int v = 0; v < out[h].nv; ++v)
            for (int k = 0; k < 3; ++k) out[h].v[v].nbr[k] = side[out[h].v[v].nbr[k]];
}

/* Moments of the polyhedron in q-space, orders 0..2 (1, 4 or 10 values), by
 * fan-triangulating every face (src/geometry.c:692-767). */
static void ov_reduce(const ov_poly *P, ov_real *mom, int order)
{
    static const int nmom[3] = {1, 4, 10};
    unsigned char done[OV_MAXV][3];
    for (int i = 0; i < nmom[order]; ++i) mom[i] = 0;
    memset(done, 0, sizeof(done));
    for (int vs = 0; vs < P->nv; ++vs)
        for (int ks = 0; ks < 3; ++ks) {
            if (done[vs][ks]) continue;
            int vc = vs, kn = ks, k;
            done[vc][kn] = 1;
            int vn = P->v[vc].nbr[kn];
            const ov_real *q0 = P->v[vc].q;
            for (k = 0; k < 3; ++k)
                if (P->v[vn].nbr[k] == vc) break;
            vc = vn;
            kn = (k + 1) % 3;
            done[vc][kn] = 1;
            vn = P->v[vc].nbr[kn];
            int steps = 0;
            while (vn != vs) {
                if (++steps > OV_WALK_CAP) { g_cnt->errors++; return; }
                const ov_real *q1 = P->v[vn].q;
                const ov_real *q2 = P->v[vc].q;
                /* 6 x signed volume of the cone (0, q0, q1, q2) */
                ov_real m = (-q2[0] * q1[1] * q0[2] + q1[0] * q2[1] * q0[2] + q2[0] * q0[1] * q1[2]
                            - q0[0] * q2[1] * q1[2] - q1[0] * q0[1] * q2[2] + q0[0] * q1[1] * q2[2]);
                mom[0] += m;
                if (order > 0) {
                    mom[1] += 0.25 * m * (q0[0] + q1[0] + q2[0]);
                    mom[2] += 0.25 * m * (q0[1] + q1[1] + q2[1]);
                    mom[3] += 0.25 * m * (q0[2] + q1[2] + q2[2]);
                }
                if (order > 1) {
                    mom[4] += ((ov_real)1 / 10) * m * (q0[0] * q0[0] + q1[0] * q1[0] + q2[0] * q2[0] + q1[0] * q2[0] + q0[0] * (q1[0] + q2[0]));
                    mom[5] += ((ov_real)1 / 20) * m * (q2[0] * q0[1] + q2[0] * q1[1] + 2 * q2[0] * q2[1] + q0[0] * (2 * q0[1] + q1[1] + q2[1]) + q1[0] * (q0[1] + 2 * q1[1] + q2[1]));
                    mom[6] += ((ov_real)1 / 20) * m * (q2[0] * q0[2] + q2[0] * q1[2] + 2 * q2[0] * q2[2] + q0[0] * (2 * q0[2] + q1[2] + q2[2]) + q1[0] * (q0[2] + 2 * q1[2] + q2[2]));
                    mom[7] += ((ov_real)1 / 10) * m * (q0[1] * q0[1] + q1[1] * q1[1] + q2[1] * q2[1] + q1[1] * q2[1] + q0[1] * (q1[1] + q2[1]));
                    mom[8] += ((ov_real)1 / 20) * m * (q2[1] * q0[2] + q2[1] * q1[2] + 2 * q2[1] * q2[2] + q0[1] * (2 * q0[2] + q1[2] + q2[2]) + q1[1] * (q0[2] + 2 * q1[2] + q2[2]));
                    mom[9] += ((ov_real)1 / 10) * m * (q0[2] * q0[2] + q1[2] * q1[2] + q2[2] * q2[2] + q1[2] * q2[2] + q0[2] * (q1[2] + q2[2]));
                }
                for (k = 0; k < 3; ++k)
                    if (P->v[vn].nbr[k] == vc) break;
                vc = vn;
                kn = (k + 1) % 3;
                done[vc][kn] = 1;
                vn = P->v[vc].nbr[kn];
            }
        }
}

/* The tet as a vertex graph with q = (0, e_x, e_y, e_z) (src/geometry.c:769-804). */
static void ov_init_tet(ov_poly *P, const double (*pos)[3])
{
    static const int nb[4][3] = {{1, 3, 2}, {2, 3, 0}, {0, 3, 1}, {1, 2, 0}};
    memset(P, 0, sizeof(*P));
    P->nv = 4;
    for (int v = 0; v < 4; ++v) {
        for (int k = 0; k < 3; ++k) P->v[v].nbr[k] = nb[v][k];
        for (int i = 0; i < 3; ++i) P->v[v].pos[i] = pos[v][i];
    }
    P->v[1].q[0] = 1.0;
    P->v[2].q[1] = 1.0;
    P->v[3].q[2] = 1.0;
}

/* Deposit one tet image on the grid: window clip, index box, bisection to
 * single voxels, moment projection and the online field update
 * (src/geometry.c:60-188, :806-896). */
static void ov_voxelize_tet(const double (*pos)[3], const double (*vel)[3], double mass,
                            const double (*rbox)[3], const og_grid *g, ov_poly *stack)
{
    static const int qi[3][3] = {{4, 5, 6}, {5, 7, 8}, {6, 8, 9}};
    ov_real DX[3][3], DV[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            DX[i][j] = pos[j + 1][i] - pos[0][i];
            DV[i][j] = vel[j + 1][i] - vel[0][i];
        }
    int order = 0;
    if (g->f[1] || g->f[2]) order = 1;
    if (g->f[3] || g->f[4] || g->f[5]) order = 2;

    ov_poly *P = &stack[0];
    ov_init_tet(P, pos);

    /* window planes and index box (src/geometry.c:806-843) */
    ov_real pn[6][3], pd[6];
    int npl = 0;
    memset(pn, 0, sizeof(pn));
    memset(pd, 0, sizeof(pd));
    for (int i = 0; i < 3; ++i) {
        double cmin = rbox[0][i], cmax = rbox[1][i];
        int clo = 0, chi = 0;
        if (g->win[0][i] > cmin) { cmin = g->win[0][i]; clo = 1; }
        if (g->win[1][i] < cmax) { cmax = g->win[1][i]; chi = 1; }
        if (clo) { pn[npl][i] = 1.0; pd[npl] = -cmin; npl++; }
        if (chi) { pn[npl][i] = -1.0; pd[npl] = cmax; npl++; }
        P->lo[i] = (int)floor((cmin - g->win[0][i]) / g->d[i]);
        P->hi[i] = (int)ceil((cmax - g->win[0][i]) / g->d[i]);
        if (P->lo[i] < 0) P->lo[i] = 0;
        if (P->hi[i] > g->n[i]) P->hi[i] = g->n[i];
    }
    note_nv(P->nv);
    ov_clip(P, (const ov_real(*)[3])pn, pd, npl);

    int top = 1;
    ov_poly cur;
    ov_real mom[10];
    while (top > 0) {
        cur = stack[--top];
        if (cur.nv <= 0) continue;
        int dmax = 0, ax = 0;
        for (int i = 0; i < 3; ++i) {
            int sz = cur.hi[i] - cur.lo[i];
            if (sz > dmax) { dmax = sz; ax = i; }
        }
        if (dmax <= 1) {
            /* dmax == 0 only for a tet image collapsed onto grid planes in every
             * axis; the reference loops forever there, this oracle reduces it. */
            ov_reduce(&cur, mom, order);
            if (mom[0] <= 0.0) continue;
            if (cur.lo[0] >= g->n[0] || cur.lo[1] >= g->n[1] || cur.lo[2] >= g->n[2]) {
                g_cnt->errors++;
                continue;
            }
            long long gi = (long long)g->n[1] * g->n[2] * cur.lo[0] + (long long)g->n[2] * cur.lo[1] + cur.lo[2];
            g_cnt->fragments++;
            g_cnt->frag_verts += cur.nv;

            ov_real cm[3], cv[3], sxx[3][3], sxv[3][3], svv[3][3];
            if (g->f[1])
                for (int i = 0; i < 3; ++i) {
                    cm[i] = mom[0] * pos[0][i];
                    for (int j = 0; j < 3; ++j) cm[i] += mom[j + 1] * DX[i][j];
                    cm[i] /= mom[0];
                }
            if (g->f[2])
                for (int i = 0; i < 3; ++i) {
                    cv[i] = mom[0] * vel[0][i];
                    for (int j = 0; j < 3; ++j) cv[i] += mom[j + 1] * DV[i][j];
                    cv[i] /= mom[0];
                }
            if (g->f[3])
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        sxx[i][j] = mom[0] * (pos[0][i] - cm[i]) * (pos[0][j] - cm[j]);
                        for (int a = 0; a < 3; ++a) {
                            sxx[i][j] += DX[i][a] * mom[1 + a] * (pos[0][j] - cm[j]);
                            sxx[i][j] += DX[j][a] * mom[1 + a] * (pos[0][i] - cm[i]);
                        }
                        for (int a = 0; a < 3; ++a)
                            for (int b = 0; b < 3; ++b) sxx[i][j] += DX[i][a] * DX[j][b] * mom[qi[a][b]];
                        sxx[i][j] /= mom[0];
                    }
            if (g->f[4])
                /* the reference pairs DX with (x0 - cm) and DV with (v0 - cv)
                 * in the two cross terms (src/geometry.c:139-140); kept as is */
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        sxv[i][j] = mom[0] * (pos[0][i] - cm[i]) * (vel[0][j] - cv[j]);
                        for (int a = 0; a < 3; ++a) {
                            sxv[i][j] += DX[i][a] * mom[1 + a] * (pos[0][j] - cm[j]);
                            sxv[i][j] += DV[j][a] * mom[1 + a] * (vel[0][i] - cv[i]);
                        }
                        for (int a = 0; a < 3; ++a)
                            for (int b = 0; b < 3; ++b) sxv[i][j] += DX[i][a] * DV[j][b] * mom[qi[a][b]];
                        sxv[i][j] /= mom[0];
                    }
            if (g->f[5])
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        svv[i][j] = mom[0] * (vel[0][i] - cv[i]) * (vel[0][j] - cv[j]);
                        for (int a = 0; a < 3; ++a) {
                            svv[i][j] += DV[i][a] * mom[1 + a] * (vel[0][j] - cv[j]);
                            svv[i][j] += DV[j][a] * mom[1 + a] * (vel[0][i] - cv[i]);
                        }
                        for (int a = 0; a < 3; ++a)
                            for (int b = 0; b < 3; ++b) svv[i][j] += DV[i][a] * DV[j][b] * mom[qi[a][b]];
                        svv[i][j] /= mom[0];
                    }

            /* online weighted update (src/geometry.c:164-186) */
            double *M = g->f[0], *X = g->f[1], *V = g->f[2];
            ov_real cw = mass * mom[0] / (M[gi] + mass * mom[0]);
            ov_real dw = M[gi] / (M[gi] + mass * mom[0]);
            if (g->f[3])
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        double *t = &g->f[3][9 * gi + 3 * i + j];
                        *t = dw * *t + cw * sxx[i][j] + cw * dw * (cm[i] - X[3 * gi + i]) * (cm[j] - X[3 * gi + j]);
                    }
            if (g->f[4])
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        double *t = &g->f[4][9 * gi + 3 * i + j];
                        *t = dw * *t + cw * sxv[i][j] + cw * dw * (cm[i] - X[3 * gi + i]) * (cv[j] - V[3 * gi + j]);
                    }
            if (g->f[5])
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        double *t = &g->f[5][9 * gi + 3 * i + j];
                        *t = dw * *t + cw * svv[i][j] + cw * dw * (cv[i] - V[3 * gi + i]) * (cv[j] - V[3 * gi + j]);
                    }
            if (X)
                for (int i = 0; i < 3; ++i) X[3 * gi + i] += cw * (cm[i] - X[3 * gi + i]);
            if (V)
                for (int i = 0; i < 3; ++i) V[3 * gi + i] += cw * (cv[i] - V[3 * gi + i]);
            M[gi] += mass * mom[0];
            continue;
        }
        if (top + 2 > OV_STACK) { g_cnt->errors++; continue; }
        double coord = g->d[ax] * (cur.lo[ax] + dmax / 2) + g->win[0][ax];
        ov_split(&cur, &stack[top], coord, ax);
        memcpy(stack[top].lo, cur.lo, sizeof(cur.lo));
        memcpy(stack[top].hi, cur.hi, sizeof(cur.hi));
        stack[top].hi[ax] -= dmax - dmax / 2;
        memcpy(stack[top + 1].lo, cur.lo, sizeof(cur.lo));
        memcpy(stack[top + 1].hi, cur.hi, sizeof(cur.hi));
        stack[top + 1].lo[ax] += dmax / 2;
        top += 2;
    }
}

/* ---- element -> tets (src/refine.c) ---- */

typedef struct {
    double (*pos)[3]; /* 4 per tet */
    double (*vel)[3];
    double *mass;
    int num, cap;
    int max_lvl;
    double ptol2;
    int mode;          /* 0: the reference's midpoint test; 1: the stretch test (not in the reference) */
    double stretch, lag[3];
} ov_tetbuf;

static const int TET_CORNERS[6][4] = {{2, 0, 6, 18}, {8, 2, 6, 18}, {8, 20, 2, 18},
                                      {8, 24, 20, 18}, {8, 6, 24, 18}, {8, 26, 20, 24}}; /* src/refine.c:39-41 */
#define I2(a, b, c) (4 * (a) + 2 * (b) + (c))
#define I3(a, b, c) (9 * (a) + 3 * (b) + (c))

static int tetbuf_reserve(ov_tetbuf *tb, int extra)
{
    if (tb->num + extra > tb->cap) {
        int nc = tb->cap ? 2 * tb->cap : 64;
        while (nc < tb->num + extra) nc *= 2;
        void *a = realloc(tb->pos, (size_t)nc * 4 * sizeof(*tb->pos));
        if (!a) return -1;
        tb->pos = a;
        a = realloc(tb->vel, (size_t)nc * 4 * sizeof(*tb->vel));
        if (!a) return -1;
        tb->vel = a;
        a = realloc(tb->mass, (size_t)nc * sizeof(double));
        if (!a) return -1;
        tb->mass = a;
        tb->cap = nc;
    }
    return 0;
}

static int tetbuf_push6(ov_tetbuf *tb, const double (*p)[3], const double (*u)[3], double mass)
{
    if (tetbuf_reserve(tb, 6)) return -1;
    for (int t = 0; t < 6; ++t) {
        for (int v = 0; v < 4; ++v) {
            int c = TET_CORNERS[t][v];
            memcpy(tb->pos[4 * tb->num + v], p[c], 3 * sizeof(double));
            memcpy(tb->vel[4 * tb->num + v], u[c], 3 * sizeof(double));
        }
        tb->mass[tb->num] = mass * (1.0 / 6); /* M_PER_TET, src/refine.c:49,147 */
        tb->num++;
    }
    return 0;
}

/* 8 cube corners -> 27 nodes by repeated midpoints (src/refine.c:292-319). */
static void interp_trilinear(const double (*in)[3], double (*out)[3])
{
    for (int ax = 0; ax < 3; ++ax) {
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j)
                for (int k = 0; k < 2; ++k) out[I3(2 * i, 2 * j, 2 * k)][ax] = in[I2(i, j, k)][ax];
        for (int j = 0; j < 3; j += 2)
            for (int k = 0; k < 3; k += 2)
                out[I3(1, j, k)][ax] = 0.5 * (out[I3(0, j, k)][ax] + out[I3(2, j, k)][ax]);
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < 3; k += 2)
                out[I3(i, 1, k)][ax] = 0.5 * (out[I3(i, 0, k)][ax] + out[I3(i, 2, k)][ax]);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                out[I3(i, j, 1)][ax] = 0.5 * (out[I3(i, j, 0)][ax] + out[I3(i, j, 2)][ax]);
    }
}

/* Adaptive octree refinement of a trilinear element (src/refine.c:223-289). */
/* EXTENSION, not in the reference: refine a (sub)cube of level lvl whose edge
 * along axis a is longer than T lag_a / 2^lvl, or whose volume (sum of the
 * |volume| of its six tets) exceeds T lag_x lag_y lag_z / 8^lvl.  The GPU
 * tessellation (stretch_refine) states the same test in the same order. */
static int stretch_refine(const double (*p)[3], int lvl, double T, const double *lag)
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
                if (d2 > lim * lim) return 1;
            }
    }
    double vol = 0.0;
    for (int t = 0; t < 6; ++t) {
        const double *q0 = p[TET_CORNERS[t][0]];
        double e[3][3];
        for (int v = 0; v < 3; ++v)
            for (int c = 0; c < 3; ++c) e[v][c] = p[TET_CORNERS[t][v + 1]][c] - q0[c];
        const double det = e[0][0] * (e[1][1] * e[2][2] - e[1][2] * e[2][1]) -
                           e[0][1] * (e[1][0] * e[2][2] - e[1][2] * e[2][0]) +
                           e[0][2] * (e[1][0] * e[2][1] - e[1][1] * e[2][0]);
        vol += fabs(det);
    }
    return vol / 6.0 > T * lag[0] * lag[1] * lag[2] * (s * s * s);
}

static int refine_trilinear(ov_tetbuf *tb, const double (*p)[3], const double (*u)[3], double mass, int lvl)
{
    static const int edges[7][3] = {{2, 4, 6}, {2, 10, 18}, {6, 12, 18}, {8, 13, 18},
                                    {8, 14, 20}, {8, 16, 24}, {20, 22, 24}};
    if (lvl < tb->max_lvl)
        for (int e = 0; e < 7; ++e) {
            int refine;
            if (tb->mode == 1) {
                refine = e == 0 && stretch_refine(p, lvl, tb->stretch, tb->lag);
            } else {
                double err2 = 0.0;
                for (int i = 0; i < 3; ++i) {
                    double mt = 0.5 * (p[edges[e][0]][i] + p[edges[e][2]][i]);
                    double ml = p[edges[e][1]][i];
                    err2 += (mt - ml) * (mt - ml);
                }
                refine = err2 > tb->ptol2;
            }
            if (refine) {
                double cp[8][3], cu[8][3], np_[27][3], nu[27][3];
                for (int i = 0; i < 2; ++i)
                    for (int j = 0; j < 2; ++j)
                        for (int k = 0; k < 2; ++k) {
                            for (int a = 0; a < 2; ++a)
                                for (int b = 0; b < 2; ++b)
                                    for (int c = 0; c < 2; ++c) {
                                        memcpy(cp[I2(a, b, c)], p[I3(a + i, b + j, c + k)], sizeof(cp[0]));
                                        memcpy(cu[I2(a, b, c)], u[I3(a + i, b + j, c + k)], sizeof(cu[0]));
                                    }
                            interp_trilinear((const double(*)[3])cp, np_);
                            interp_trilinear((const double(*)[3])cu, nu);
                            if (refine_trilinear(tb, (const double(*)[3])np_, (const double(*)[3])nu, 0.125 * mass, lvl + 1))
                                return -1;
                        }
                return 0;
            }
        }
    return tetbuf_push6(tb, p, u, mass);
}

/* Triquadratic elements (27 nodes, index 9i+3j+k): the 125-node interpolation of
 * src/refine.c:321-345 -- the corner values at even lattice points, then three
 * sweeps (x on the even y, z planes; y on the even z planes; z everywhere), each
 * new node 1/8 (3 near + 6 middle - far) of the three nodes of its line. */
#define I5(a, b, c) (25 * (a) + 5 * (b) + (c))
static void quad_fill_line(double (*o)[3], int a0, int s, int ax)
{
    /* nodes a0, a0 + s, ..., a0 + 4s of one line: fill 1 and 3 from 0, 2, 4 */
    const double *n0 = o[a0], *n2 = o[a0 + 2 * s], *n4 = o[a0 + 4 * s];
    o[a0 + s][ax] = 0.125 * (3.0 * n0[ax] + 6.0 * n2[ax] - n4[ax]);
    o[a0 + 3 * s][ax] = 0.125 * (3.0 * n4[ax] + 6.0 * n2[ax] - n0[ax]);
}

static void interp_triquadratic(const double (*in)[3], double (*out)[3])
{
    for (int ax = 0; ax < 3; ++ax) {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) out[I5(2 * i, 2 * j, 2 * k)][ax] = in[I3(i, j, k)][ax];
        for (int j = 0; j < 5; j += 2)
            for (int k = 0; k < 5; k += 2) quad_fill_line(out, I5(0, j, k), 25, ax);
        for (int i = 0; i < 5; ++i)
            for (int k = 0; k < 5; k += 2) quad_fill_line(out, I5(i, 0, k), 5, ax);
        for (int i = 0; i < 5; ++i)
            for (int j = 0; j < 5; ++j) quad_fill_line(out, I5(i, j, 0), 1, ax);
    }
}

/* src/refine.c:152-221: refine while the midpoint of one of the 19 tet edges of
 * the 3x3x3 node cube (end, midpoint, end: the table of src/refine.c:157-161)
 * deviates from the straight edge by more than the tolerance; child (i,j,k)
 * takes nodes (2i..2i+2, ...) of the 125-node interpolation; a leaf is the six
 * tets of its corner nodes. */
static int refine_triquadratic(ov_tetbuf *tb, const double (*p)[3], const double (*u)[3], double mass, int lvl)
{
    static const int edges[19][3] = {{0, 1, 2},    {0, 3, 6},    {0, 9, 18},   {2, 4, 6},    {2, 5, 8},
                                     {2, 10, 18},  {2, 11, 20},  {6, 7, 8},    {6, 12, 18},  {6, 15, 24},
                                     {8, 13, 18},  {8, 14, 20},  {8, 16, 24},  {8, 17, 26},  {18, 19, 20},
                                     {18, 21, 24}, {20, 22, 24}, {20, 23, 26}, {24, 25, 26}};
    if (lvl < tb->max_lvl)
        for (int e = 0; e < 19; ++e) {
            double err2 = 0.0;
            for (int i = 0; i < 3; ++i) {
                double mt = 0.5 * (p[edges[e][0]][i] + p[edges[e][2]][i]);
                double mq = p[edges[e][1]][i];
                err2 += (mt - mq) * (mt - mq);
            }
            if (err2 > tb->ptol2) {
                double ip[125][3], iu[125][3], cp[27][3], cu[27][3];
                interp_triquadratic(p, ip);
                interp_triquadratic(u, iu);
                for (int i = 0; i < 2; ++i)
                    for (int j = 0; j < 2; ++j)
                        for (int k = 0; k < 2; ++k) {
                            for (int a = 0; a < 3; ++a)
                                for (int b = 0; b < 3; ++b)
                                    for (int c = 0; c < 3; ++c) {
                                        memcpy(cp[I3(a, b, c)], ip[I5(a + 2 * i, b + 2 * j, c + 2 * k)], sizeof(cp[0]));
                                        memcpy(cu[I3(a, b, c)], iu[I5(a + 2 * i, b + 2 * j, c + 2 * k)], sizeof(cu[0]));
                                    }
                            if (refine_triquadratic(tb, (const double(*)[3])cp, (const double(*)[3])cu, 0.125 * mass,
                                                    lvl + 1))
                                return -1;
                        }
                return 0;
            }
        }
    return tetbuf_push6(tb, p, u, mass);
}

/* An element's tets into tb (src/refine.c:58-150): a simplex is one tet of the
 * element's mass, a trilinear or triquadratic element is refined. */
static int element_tets(ov_tetbuf *tb, const double (*p)[3], const double (*u)[3], double mass, int vpe)
{
    tb->num = 0;
    if (vpe == 4) {
        if (tetbuf_reserve(tb, 1)) return -1;
        memcpy(tb->pos[0], p, sizeof(double) * 12);
        memcpy(tb->vel[0], u, sizeof(double) * 12);
        tb->mass[0] = mass;
        tb->num = 1;
        return 0;
    }
    if (vpe == 27) return refine_triquadratic(tb, p, u, mass, 0); /* the 27 nodes as they are (src/refine.c:79-81) */
    double np_[27][3], nu[27][3];
    interp_trilinear(p, np_);
    interp_trilinear(u, nu);
    return refine_trilinear(tb, (const double(*)[3])np_, (const double(*)[3])nu, mass, 0);
}

/* ---- element loop helpers (src/cpsi.c:277-373) ---- */

static void aabb(const double (*p)[3], int n, double (*rb)[3])
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

static int aabb_periodic(double (*p)[3], int n, double (*rb)[3], const og_grid *g, const og_mesh *m)
{
    aabb((const double(*)[3])p, n, rb);
    if (m->periodic) {
        for (int i = 0; i < 3; ++i) {
            double span = m->box[1][i] - m->box[0][i];
            if (rb[1][i] - rb[0][i] > 0.5 * span) {
                rb[0][i] = 1.0e30;
                rb[1][i] = -1.0e30;
                for (int v = 0; v < n; ++v) {
                    if (p[v][i] > m->box[0][i] + 0.5 * span) p[v][i] -= span;
                    if (p[v][i] < rb[0][i]) rb[0][i] = p[v][i];
                    if (p[v][i] > rb[1][i]) rb[1][i] = p[v][i];
                }
            }
            if (rb[0][i] > g->win[1][i]) return 0;
            if (rb[1][i] < g->win[0][i] && rb[0][i] + span > g->win[1][i]) return 0;
        }
    } else {
        for (int i = 0; i < 3; ++i) {
            if (rb[0][i] > g->win[1][i]) return 0;
            if (rb[1][i] < g->win[0][i]) return 0;
        }
    }
    return 1;
}

/* Up to 8 periodic images of a tet (src/cpsi.c:343-373). */
static int make_images(double (*p)[3], double (*rb)[3], const og_grid *g, const og_mesh *m)
{
    int num = 1, flags = 0;
    double span[3];
    if (!m->periodic) return 1;
    for (int i = 0; i < 3; ++i) {
        span[i] = m->box[1][i] - m->box[0][i];
        if (rb[0][i] < m->box[0][i]) flags |= 1 << i;
    }
    for (int s = 1; s < 8; ++s) {
        if ((flags & s) != s) continue;
        int ok = 1;
        for (int i = 0; i < 3 && ok; ++i) {
            double sh = span[i] * (1 & (s >> i));
            rb[2 * num + 0][i] = rb[0][i] + sh;
            rb[2 * num + 1][i] = rb[1][i] + sh;
            if (rb[2 * num + 0][i] > g->win[1][i] || rb[2 * num + 1][i] < g->win[0][i]) {
                ok = 0;
                break;
            }
            for (int v = 0; v < 4; ++v) p[4 * num + v][i] = p[v][i] + sh;
        }
        if (ok) num++;
    }
    return num;
}

/* The density branch of psi_voxels (src/cpsi.c:41-112).  Returns 0, or -1 on
 * an unsupported element type / allocation failure. */
static int voxels_impl(og_grid *g, const og_mesh *m, double reftol, int max_lvl, int mode, const double *lag,
                       og_counters *cnt);

int oracle_voxels(og_grid *g, const og_mesh *m, double reftol, int max_lvl, og_counters *cnt)
{
    return voxels_impl(g, m, reftol, max_lvl, 0, NULL, cnt);
}

/* With the refinement criterion of the GPU library's PSIB_REFINE_STRETCH
 * (mode 1, threshold reftol, Lagrangian cell lag). */
int oracle_voxels_ex(og_grid *g, const og_mesh *m, double reftol, int max_lvl, int mode, const double *lag,
                     og_counters *cnt)
{
    return voxels_impl(g, m, reftol, max_lvl, mode, lag, cnt);
}

static int voxels_impl(og_grid *g, const og_mesh *m, double reftol, int max_lvl, int mode, const double *lag,
                       og_counters *cnt)
{
    og_counters dummy;
    memset(&dummy, 0, sizeof(dummy));
    g_cnt = cnt ? cnt : &dummy;
    if (m->elemtype != 4 && m->elemtype != 8 && m->elemtype != 27) return -1;
    double dxmin = 1.0e30;
    for (int i = 0; i < 3; ++i)
        if (g->d[i] < dxmin) dxmin = g->d[i];
    ov_tetbuf tb;
    memset(&tb, 0, sizeof(tb));
    if (max_lvl > 6) max_lvl = 6; /* src/refine.c:89-92 */
    tb.max_lvl = max_lvl;
    tb.ptol2 = (reftol * dxmin) * (reftol * dxmin);
    tb.mode = mode;
    tb.stretch = reftol;
    for (int i = 0; i < 3; ++i) tb.lag[i] = lag ? lag[i] : 0.0;
    ov_poly *stack = malloc(OV_STACK * sizeof(ov_poly));
    if (!stack) return -1;
    int vpe = m->elemtype;
    int rc = 0;
    for (int e = 0; e < m->nelem; ++e) {
        double tp[27][3], tu[27][3], rb[2][3];
        for (int v = 0; v < vpe; ++v) {
            int id = m->conn[e * vpe + v];
            memcpy(tp[v], &m->pos[3 * (size_t)id], sizeof(tp[v]));
            memcpy(tu[v], &m->vel[3 * (size_t)id], sizeof(tu[v]));
        }
        if (!aabb_periodic(tp, vpe, rb, g, m)) continue;
        g_cnt->elements_kept++;
        if (element_tets(&tb, (const double(*)[3])tp, (const double(*)[3])tu, m->mass[e], vpe)) { rc = -1; break; }
        for (int t = 0; t < tb.num; ++t) {
            double gp[32][3], grb[16][3];
            memcpy(gp, tb.pos[4 * t], sizeof(double) * 12);
            aabb((const double(*)[3])gp, 4, grb);
            int ng = make_images(gp, grb, g, m);
            g_cnt->tets++;
            for (int k = 0; k < ng; ++k) {
                g_cnt->tet_images++;
                ov_voxelize_tet((const double(*)[3])&gp[4 * k], (const double(*)[3])tb.vel[4 * t], tb.mass[t],
                                (const double(*)[3])&grb[2 * k], g, stack);
            }
        }
    }
    free(stack);
    free(tb.pos);
    free(tb.vel);
    free(tb.mass);
    return rc;
}

/* ---- annihilation mode (src/cpsi.c:115-158, src/geometry.c:190-252) ----
 *
 * For every element e that survives the window cull (its vertices unwrapped,
 * src/cpsi.c:309-341), every element e1 that survives it too and whose
 * unwrapped box touches e's (closed intervals: the R*-tree query of
 * src/rtree.c:83-125), every tet t of e (refined from the unwrapped vertices)
 * and every tet t1 of e1 (refined from e1's vertices as stored, without the
 * unwrap, src/cpsi.c:123-131) whose boxes overlap with positive extent
 * (src/cpsi.c:293-306): the intersection of t and t1 deposits
 * rho_t rho_t1 x (its volume in each voxel) into m.
 *
 * The reference visits e1 in the depth-first order of its R*-tree.  With at
 * most 32 surviving elements that tree is one leaf holding them in index order,
 * whose query returns them last first; this restatement takes that order
 * (descending e1) for every mesh, so it equals the reference bit for bit up to
 * 32 surviving elements and to rounding beyond. */

static ov_real ov_third(void) { return (ov_real)1 / 3; }

/* psi_orient_tet (src/geometry.c:190-224): six times the signed volume is the
 * triple product of the edges from vertex 3, expanded as
 * a.x (b x c).x + b.x (c x a).x + c.x (a x b).x; a negative tet has vertices
 * 0 and 1 swapped.  Returns the volume. */
static ov_real orient_tet(double (*p)[3])
{
    ov_real a[3], b[3], c[3];
    for (int i = 0; i < 3; ++i) {
        a[i] = (ov_real)p[0][i] - p[3][i];
        b[i] = (ov_real)p[1][i] - p[3][i];
        c[i] = (ov_real)p[2][i] - p[3][i];
    }
    const ov_real s = a[0] * (b[1] * c[2] - b[2] * c[1]) + b[0] * (c[1] * a[2] - c[2] * a[1]) +
                      c[0] * (a[1] * b[2] - a[2] * b[1]);
    ov_real vol = -((ov_real)1 / 6) * s;
    if (vol < 0.0) {
        for (int i = 0; i < 3; ++i) {
            double t = p[0][i];
            p[0][i] = p[1][i];
            p[1][i] = t;
        }
        vol = -vol;
    }
    return vol;
}

/* One face plane n.x + d >= 0 of a tet (src/geometry.c:503-558): n = A x B of
 * the two edge vectors A = a1 - a0, B = b1 - b0 the reference uses for that
 * face, d = -n . (third of the sum of the face's vertices f0 + f1 + f2). */
static void face_plane(const double *a0, const double *a1, const double *b0, const double *b1, const double *f0,
                       const double *f1, const double *f2, ov_real *n, ov_real *d)
{
    ov_real A[3], B[3], c[3];
    for (int i = 0; i < 3; ++i) {
        A[i] = (ov_real)a1[i] - a0[i];
        B[i] = (ov_real)b1[i] - b0[i];
        c[i] = ov_third() * ((ov_real)f0[i] + f1[i] + f2[i]);
    }
    n[0] = A[1] * B[2] - A[2] * B[1];
    n[1] = A[2] * B[0] - A[0] * B[2];
    n[2] = A[0] * B[1] - A[1] * B[0];
    *d = -(n[0] * c[0] + n[1] * c[1] + n[2] * c[2]);
}

static void tet_faces(const double (*v)[3], ov_real (*n)[3], ov_real *d)
{
    face_plane(v[1], v[3], v[1], v[2], v[1], v[2], v[3], n[0], &d[0]);
    face_plane(v[0], v[2], v[2], v[3], v[2], v[3], v[0], n[1], &d[1]);
    face_plane(v[3], v[1], v[3], v[0], v[3], v[0], v[1], n[2], &d[2]);
    face_plane(v[2], v[0], v[0], v[1], v[0], v[1], v[2], n[3], &d[3]);
}

/* psi_voxelize_annihilation (src/geometry.c:226-252) of two oriented tets. */
static void ov_annihilate(const double (*p0)[3], ov_real vol0, ov_real rho0, const double (*p1)[3], ov_real rho1,
                          const double (*mbox)[3], const og_grid *g, ov_poly *stack)
{
    ov_poly *P = &stack[0];
    ov_init_tet(P, p0);
    ov_real fn[4][3], fd[4];
    tet_faces(p1, fn, fd);
    ov_clip(P, (const ov_real(*)[3])fn, fd, 4);

    ov_real pn[6][3], pd[6];
    int npl = 0;
    memset(pn, 0, sizeof(pn));
    memset(pd, 0, sizeof(pd));
    for (int i = 0; i < 3; ++i) {
        double cmin = mbox[0][i], cmax = mbox[1][i];
        int clo = 0, chi = 0;
        if (g->win[0][i] > cmin) { cmin = g->win[0][i]; clo = 1; }
        if (g->win[1][i] < cmax) { cmax = g->win[1][i]; chi = 1; }
        if (clo) { pn[npl][i] = 1.0; pd[npl] = -cmin; npl++; }
        if (chi) { pn[npl][i] = -1.0; pd[npl] = cmax; npl++; }
        P->lo[i] = (int)floor((cmin - g->win[0][i]) / g->d[i]);
        P->hi[i] = (int)ceil((cmax - g->win[0][i]) / g->d[i]);
        if (P->lo[i] < 0) P->lo[i] = 0;
        if (P->hi[i] > g->n[i]) P->hi[i] = g->n[i];
    }
    note_nv(P->nv);
    ov_clip(P, (const ov_real(*)[3])pn, pd, npl);

    const ov_real w = rho0 * rho1 * vol0;
    int top = 1;
    ov_poly cur;
    ov_real mom[10];
    while (top > 0) {
        cur = stack[--top];
        if (cur.nv <= 0) continue;
        int dmax = 0, ax = 0;
        for (int i = 0; i < 3; ++i) {
            int sz = cur.hi[i] - cur.lo[i];
            if (sz > dmax) { dmax = sz; ax = i; }
        }
        if (dmax <= 1) {
            ov_reduce(&cur, mom, 0);
            if (mom[0] <= 0.0) continue;
            if (cur.lo[0] >= g->n[0] || cur.lo[1] >= g->n[1] || cur.lo[2] >= g->n[2]) {
                g_cnt->errors++;
                continue;
            }
            long long gi = (long long)g->n[1] * g->n[2] * cur.lo[0] + (long long)g->n[2] * cur.lo[1] + cur.lo[2];
            g_cnt->fragments++;
            g_cnt->frag_verts += cur.nv;
            g->f[0][gi] += w * mom[0];
            continue;
        }
        if (top + 2 > OV_STACK) { g_cnt->errors++; continue; }
        double coord = g->d[ax] * (cur.lo[ax] + dmax / 2) + g->win[0][ax];
        ov_split(&cur, &stack[top], coord, ax);
        memcpy(stack[top].lo, cur.lo, sizeof(cur.lo));
        memcpy(stack[top].hi, cur.hi, sizeof(cur.hi));
        stack[top].hi[ax] -= dmax - dmax / 2;
        memcpy(stack[top + 1].lo, cur.lo, sizeof(cur.lo));
        memcpy(stack[top + 1].hi, cur.hi, sizeof(cur.hi));
        stack[top + 1].lo[ax] += dmax / 2;
        top += 2;
    }
}

int oracle_annihilation(og_grid *g, const og_mesh *m, double reftol, int max_lvl, og_counters *cnt)
{
    og_counters dummy;
    memset(&dummy, 0, sizeof(dummy));
    g_cnt = cnt ? cnt : &dummy;
    if (m->elemtype != 4 && m->elemtype != 8 && m->elemtype != 27) return -1;
    const int vpe = m->elemtype;
    double dxmin = 1.0e30;
    for (int i = 0; i < 3; ++i)
        if (g->d[i] < dxmin) dxmin = g->d[i];
    if (max_lvl > 6) max_lvl = 6;
    ov_tetbuf ta, tb;
    memset(&ta, 0, sizeof(ta));
    memset(&tb, 0, sizeof(tb));
    ta.max_lvl = tb.max_lvl = max_lvl;
    ta.ptol2 = tb.ptol2 = (reftol * dxmin) * (reftol * dxmin);
    double(*box)[2][3] = malloc((size_t)(m->nelem > 0 ? m->nelem : 1) * sizeof(*box));
    char *kept = calloc((size_t)(m->nelem > 0 ? m->nelem : 1), 1);
    ov_poly *stack = malloc(OV_STACK * sizeof(ov_poly));
    int rc = (box && kept && stack) ? 0 : -1;
    /* element boxes after the unwrap, and the cull (src/rtree.c:48-73) */
    for (int e = 0; rc == 0 && e < m->nelem; ++e) {
        double tp[27][3];
        for (int v = 0; v < vpe; ++v) memcpy(tp[v], &m->pos[3 * (size_t)m->conn[e * vpe + v]], sizeof(tp[v]));
        kept[e] = (char)aabb_periodic(tp, vpe, box[e], g, m);
    }
    for (int e = 0; rc == 0 && e < m->nelem; ++e) {
        if (!kept[e]) continue;
        g_cnt->elements_kept++;
        double tp[27][3], tu[27][3], rb[2][3];
        for (int v = 0; v < vpe; ++v) {
            int id = m->conn[e * vpe + v];
            memcpy(tp[v], &m->pos[3 * (size_t)id], sizeof(tp[v]));
            memcpy(tu[v], &m->vel[3 * (size_t)id], sizeof(tu[v]));
        }
        aabb_periodic(tp, vpe, rb, g, m);
        if (element_tets(&ta, (const double(*)[3])tp, (const double(*)[3])tu, m->mass[e], vpe)) { rc = -1; break; }
        g_cnt->tets += ta.num;
        for (int e1 = m->nelem - 1; e1 >= 0; --e1) {
            if (!kept[e1]) continue;
            int touch = 1;
            for (int i = 0; i < 3; ++i)
                if (box[e][1][i] < box[e1][0][i] || box[e][0][i] > box[e1][1][i]) touch = 0;
            if (!touch) continue;
            double sp[27][3], su[27][3];
            for (int v = 0; v < vpe; ++v) {
                int id = m->conn[e1 * vpe + v];
                memcpy(sp[v], &m->pos[3 * (size_t)id], sizeof(sp[v]));
                memcpy(su[v], &m->vel[3 * (size_t)id], sizeof(su[v]));
            }
            if (element_tets(&tb, (const double(*)[3])sp, (const double(*)[3])su, m->mass[e1], vpe)) { rc = -1; break; }
            for (int t = 0; t < ta.num; ++t) {
                double b0[2][3];
                aabb((const double(*)[3])ta.pos[4 * t], 4, b0);
                for (int t1 = 0; t1 < tb.num; ++t1) {
                    double b1[2][3], mb[2][3];
                    aabb((const double(*)[3])tb.pos[4 * t1], 4, b1);
                    int ok = 1;
                    for (int i = 0; i < 3; ++i) {
                        mb[0][i] = fmax(b0[0][i], b1[0][i]);
                        mb[1][i] = fmin(b0[1][i], b1[1][i]);
                        ok &= mb[1][i] > mb[0][i];
                    }
                    if (!ok) continue;
                    g_cnt->tet_images++;
                    /* orienting a tet in place is idempotent: each tet is oriented once */
                    ov_real vol0 = orient_tet(ta.pos + 4 * t);
                    ov_real vol1 = orient_tet(tb.pos + 4 * t1);
                    ov_real rho0 = ta.mass[t] / vol0, rho1 = tb.mass[t1] / vol1;
                    ov_annihilate((const double(*)[3])(ta.pos + 4 * t), vol0, rho0,
                                  (const double(*)[3])(tb.pos + 4 * t1), rho1, (const double(*)[3])mb, g, stack);
                }
            }
        }
    }
    free(box);
    free(kept);
    free(stack);
    free(ta.pos);
    free(ta.vel);
    free(ta.mass);
    free(tb.pos);
    free(tb.vel);
    free(tb.mass);
    return rc;
}

/* ---- element queries and phase-space samples (src/rtree.c:48-125, src/cpsi.c:177-275,
 *      src/geometry.c:335-389) ----
 *
 * The reference indexes the elements that survive the cull against a window
 * (src/rtree.c:48-73: the periodic box for PSI.RStarTree of a periodic mesh,
 * +-1e30 for an open one, the mesh's own box for the tree PSI.VDF builds when
 * given none) by their unwrapped boxes, and answers a query box with every
 * element whose box it touches (closed intervals).  This restatement scans the
 * elements in descending index: the order the reference's tree returns while
 * it is a single leaf (at most 32 elements). */

static int elem_box(const og_mesh *m, const double (*window)[3], int e, double (*rb)[3])
{
    og_grid g;
    memset(&g, 0, sizeof(g));
    memcpy(g.win, window, sizeof(g.win));
    double tp[27][3];
    for (int v = 0; v < m->elemtype; ++v) memcpy(tp[v], &m->pos[3 * (size_t)m->conn[e * m->elemtype + v]], sizeof(tp[v]));
    return aabb_periodic(tp, m->elemtype, rb, &g, m);
}

long long oracle_query(const og_mesh *m, const double (*window)[3], const double (*q)[3], int *out, long long cap)
{
    long long n = 0;
    for (int e = m->nelem - 1; e >= 0; --e) {
        double rb[2][3];
        if (!elem_box(m, window, e, rb)) continue;
        int touch = 1;
        for (int i = 0; i < 3; ++i)
            if (q[1][i] < rb[0][i] || q[0][i] > rb[1][i]) touch = 0;
        if (!touch) continue;
        if (n < cap) out[n] = e;
        n++;
    }
    return n;
}

/* psi_barycentric (src/geometry.c:335-389): the four barycentric coordinates of
 * s in the tet v (v[i] opposite coordinate i) as (w_i + s . n_i) / (their sum),
 * with w_i the signed volume term of the other three vertices -- terms
 * x_a (b x c).x summed in the reference's order -- and n_i the face normal of
 * the face opposite v[i], the same edge vectors as its face planes; returns
 * |sum| / 6, the tet's volume. */
static ov_real ov_cx(const double *a, const double *b) { return (ov_real)a[1] * b[2] - (ov_real)a[2] * b[1]; }

static void ov_cross(const double *a0, const double *a1, const double *b0, const double *b1, ov_real *n)
{
    ov_real A[3], B[3];
    for (int i = 0; i < 3; ++i) {
        A[i] = (ov_real)a1[i] - a0[i];
        B[i] = (ov_real)b1[i] - b0[i];
    }
    n[0] = A[1] * B[2] - A[2] * B[1];
    n[1] = A[2] * B[0] - A[0] * B[2];
    n[2] = A[0] * B[1] - A[1] * B[0];
}

static ov_real ov_barycentric(const double (*v)[3], const double *s, ov_real *b)
{
    ov_real w[4], n[4][3];
    w[0] = v[1][0] * ov_cx(v[2], v[3]) + v[2][0] * ov_cx(v[3], v[1]) + v[3][0] * ov_cx(v[1], v[2]);
    w[1] = v[0][0] * ov_cx(v[3], v[2]) + v[2][0] * ov_cx(v[0], v[3]) + v[3][0] * ov_cx(v[2], v[0]);
    w[2] = v[0][0] * ov_cx(v[1], v[3]) + v[1][0] * ov_cx(v[3], v[0]) + v[3][0] * ov_cx(v[0], v[1]);
    w[3] = v[0][0] * ov_cx(v[2], v[1]) + v[1][0] * ov_cx(v[0], v[2]) + v[2][0] * ov_cx(v[1], v[0]);
    ov_cross(v[1], v[3], v[1], v[2], n[0]);
    ov_cross(v[0], v[2], v[2], v[3], n[1]);
    ov_cross(v[3], v[1], v[3], v[0], n[2]);
    ov_cross(v[2], v[0], v[0], v[1], n[3]);
    ov_real tot = 0.0;
    for (int i = 0; i < 4; ++i) {
        b[i] = w[i];
        for (int j = 0; j < 3; ++j) b[i] += s[j] * n[i][j];
        tot += b[i];
    }
    for (int i = 0; i < 4; ++i) b[i] /= tot;
    ov_real vol = ((ov_real)1 / 6) * tot;
    return vol < 0 ? -vol : vol;
}

/* psi_sample_vdf (src/cpsi.c:177-275): for every element whose box contains the
 * point (a query with the degenerate box [s, s]), its tets -- refined from its
 * vertices as stored, with the tolerance reftol itself -- that contain the
 * point give one sample each: density mass / volume and the velocity
 * interpolated at the point.  Returns the number of samples; writes up to cap. */
long long oracle_sample_vdf(const og_mesh *m, const double (*window)[3], const double *s, double reftol, int max_lvl,
                            double *rho, double *vel, long long cap)
{
    static og_counters unused; /* the element refinement reports errors here */
    g_cnt = &unused;
    if (m->elemtype != 4 && m->elemtype != 8 && m->elemtype != 27) return -1;
    if (max_lvl > 6) max_lvl = 6;
    ov_tetbuf tb;
    memset(&tb, 0, sizeof(tb));
    tb.max_lvl = max_lvl;
    tb.ptol2 = reftol * reftol;
    const double q[2][3] = {{s[0], s[1], s[2]}, {s[0], s[1], s[2]}};
    long long n = 0;
    for (int e = m->nelem - 1; e >= 0; --e) {
        double rb[2][3];
        if (!elem_box(m, window, e, rb)) continue;
        int touch = 1;
        for (int i = 0; i < 3; ++i)
            if (q[1][i] < rb[0][i] || q[0][i] > rb[1][i]) touch = 0;
        if (!touch) continue;
        double tp[27][3], tu[27][3];
        for (int v = 0; v < m->elemtype; ++v) {
            int id = m->conn[e * m->elemtype + v];
            memcpy(tp[v], &m->pos[3 * (size_t)id], sizeof(tp[v]));
            memcpy(tu[v], &m->vel[3 * (size_t)id], sizeof(tu[v]));
        }
        if (element_tets(&tb, (const double(*)[3])tp, (const double(*)[3])tu, m->mass[e], m->elemtype)) {
            n = -1;
            break;
        }
        for (int t = 0; t < tb.num; ++t) {
            ov_real b[4];
            ov_real vol = ov_barycentric((const double(*)[3])tb.pos[4 * t], s, b);
            if (vol <= 0.0) continue;
            int inside = 1;
            for (int i = 0; i < 4; ++i)
                if (b[i] < 0.0) inside = 0;
            if (!inside) continue;
            if (n < cap) {
                for (int i = 0; i < 3; ++i) {
                    ov_real u = 0.0;
                    for (int j = 0; j < 4; ++j) u += b[j] * tb.vel[4 * t + j][i];
                    vel[3 * n + i] = (double)u;
                }
                rho[n] = (double)(tb.mass[t] / vol);
            }
            n++;
        }
    }
    free(tb.pos);
    free(tb.vel);
    free(tb.mass);
    return n;
}
