// noalloc.cu -- a density deposit that allocates nothing.
//
// psib_voxels allocates device buffers on its first call and grows them on
// demand.  Some callers cannot let a library do that:
//   * an application that has handed all of the GPU's memory to its own pool
//     allocator at start-up (a simulation code or another framework sharing
//     the GPU) -- a cudaMalloc from inside the library would fail, or break the
//     pool's accounting;
//   * a time-critical loop in which an allocation's implicit synchronisation
//     and latency are not acceptable.
// psib_voxels_density_noalloc serves them: it deposits the mass of tets the
// caller already holds on the device into the caller's m field, and calls no
// cudaMalloc, cudaFree or allocating library routine.  It is a variant of the
// FP64 clip kernel (the same window clip, depth-first bisection and fragment
// reduction, clip_fp64.cu / psib_clip.cuh) whose per-thread polyhedron slots
// live in the file-scope array below instead of an allocated scratch buffer,
// and which adds each fragment's mass with an atomic instead of writing a
// record for the sort-and-apply stage.
//
// Limits and sharing:
//   * The array holds NA_THREADS slot regions of NA_NS polyhedra each,
//     NA_SCRATCH_BYTES (about 7.9 MiB) in total.  Every GPU that loads the
//     library keeps it until the process exits.
//   * Depth limit: a tet is too large when the bisection of its voxel index
//     box (after the clamp to the grid window) is deeper than NA_DMAX = 12
//     levels, i.e. when sum over the three axes of ceil(log2(size_a)) > 12
//     (axes of size 1 count 0).  16x16x16 voxels (4 + 4 + 4) is accepted,
//     16x16x32 (4 + 4 + 5) rejected, 4096x1x1 (12) accepted.  A first kernel
//     checks every tet; if one is too large the call returns PSIB_ERR_ARG and
//     deposits nothing at all.
//   * Any other failure found while depositing (a polyhedron that outgrows
//     its vertex buffer, a face walk that does not close, a voxel index out of
//     range) returns PSIB_ERR_OVERFLOW or PSIB_ERR_INDEX after the other tets,
//     and part of the failing tet, have already been added to m.
//   * All calls on a device share the array and its queue and status words,
//     which keep the last call's contents; each call clears the words that
//     must start at zero.  Calls that overlap on the GPU (on different
//     streams, or from different host threads) race on them.
//   * Every call looks up the array's device address with
//     cudaGetSymbolAddress (with the caller's device current; it allocates
//     nothing), so the address stays valid after a cudaDeviceReset.  The first
//     call on a device also loads the library's kernels there and should come
//     before any stream capture.
#include <cuda_runtime.h>

#include <cstdio>

#include "psi_b200.h"
#include "psib_clip.cuh"

namespace psib {

namespace {

constexpr int NA_BLOCK = 32;                              // one warp per block: the regions spread over 16 SMs
constexpr int NA_THREADS = 16 * NA_BLOCK;                 // resident threads of one call
constexpr int NA_DMAX = 12;                               // deepest bisection served
constexpr int NA_NS = NA_DMAX + 3;                        // slots per thread
constexpr size_t NA_REGION = sizeof(Poly<double>) * NA_NS; // bytes per thread
constexpr size_t NA_STATE = 256;                          // queue head and status word
constexpr size_t NA_SCRATCH_BYTES = NA_STATE + NA_REGION * NA_THREADS;

struct NaState {
    unsigned long long head;
    unsigned status;
};

// The scratch of every call: state words first, then the per-thread regions.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_SCRATCH_BYTES];

struct NaArgs {
    const double *pos;  // ntets x 4 x 3, vertex-major
    const double *mass; // ntets (null: 1)
    long long ntets;
    GridDev g;
    double *m;
    unsigned char *scratch; // device address of g_noalloc_scratch
};

// The tet's voxel index box, clamped to the grid window (src/geometry.c:816-842).
__device__ __forceinline__ void index_box(const NaArgs& a, const double (*rb)[3], int* lo, int* hi)
{
    for (int i = 0; i < 3; ++i) {
        double cmin = rb[0][i], cmax = rb[1][i];
        if (a.g.w0[i] > cmin) cmin = a.g.w0[i];
        if (a.g.w1[i] < cmax) cmax = a.g.w1[i];
        lo[i] = (int)floor((cmin - a.g.w0[i]) / a.g.d[i]);
        hi[i] = (int)ceil((cmax - a.g.w0[i]) / a.g.d[i]);
        if (lo[i] < 0) lo[i] = 0;
        if (hi[i] > a.g.n[i]) hi[i] = a.g.n[i];
    }
}

// Depth of the box's bisection: sum over the axes of ceil(log2(size)).
__device__ __forceinline__ int box_depth(const int* lo, const int* hi)
{
    int depth = 0;
    for (int i = 0; i < 3; ++i) {
        const int sz = hi[i] - lo[i];
        if (sz > 1) depth += 32 - __clz(sz - 1);
    }
    return depth;
}

// Depth-first bisection of one tet with mass deposited by atomics.  Same
// arithmetic as clip_item<double, ..> up to the fragment's m0.
__device__ void deposit_tet(const NaArgs& a, long long t, Poly<double>* S, unsigned& st)
{
    double p[4][3];
    for (int v = 0; v < 4; ++v)
        for (int i = 0; i < 3; ++i) p[v][i] = a.pos[12 * t + 3 * v + i];
    const double mass = a.mass ? a.mass[t] : 1.0;
    double rb[2][3];
    aabb4(p, rb);
    int pax[6], psg[6], npl = 0, lo[3], hi[3];
    double pdd[6];
    for (int i = 0; i < 3; ++i) {
        double cmin = rb[0][i], cmax = rb[1][i];
        const bool clo = a.g.w0[i] > cmin, chi = a.g.w1[i] < cmax;
        if (clo) cmin = a.g.w0[i];
        if (chi) cmax = a.g.w1[i];
        if (clo) { pax[npl] = i; psg[npl] = 1; pdd[npl] = -cmin; npl++; }
        if (chi) { pax[npl] = i; psg[npl] = -1; pdd[npl] = cmax; npl++; }
    }
    index_box(a, rb, lo, hi);
    if (box_depth(lo, hi) > NA_DMAX) {
        st |= ST_DEPTH; // cannot happen after the pre-pass; kept so that no slot pool is overrun
        return;
    }
    uint32_t freem = (1u << NA_NS) - 1u;
    int8_t stk[NA_NS];
    int top = 0;
    auto alloc = [&](int& dst) {
        const int i = __ffs(freem) - 1;
        if (i < 0) return false;
        freem &= ~(1u << i);
        dst = i;
        return true;
    };
    int c;
    if (!alloc(c)) { st |= ST_OVERFLOW; return; }
    init_tet(S[c], p);
    double s[MAXV];
    for (int pl = 0; pl < npl && S[c].nv > 0; ++pl) {
        Poly<double>& P = S[c];
        const int ax = pax[pl];
        double smin = 1.0e30, smax = -1.0e30;
        uint32_t um = 0;
        for (int v = 0; v < P.nv; ++v) {
            double t0 = pdd[pl];
            for (int i = 0; i < 3; ++i) t0 += P.x[v][i] * (i == ax ? (double)psg[pl] : 0.0);
            s[v] = t0;
            if (t0 < smin) smin = t0;
            if (t0 > smax) smax = t0;
            if (t0 < 0.0) um |= 1u << v;
        }
        if (smin >= 0.0) continue;
        if (smax <= 0.0) { P.nv = 0; break; }
        int o;
        if (!alloc(o)) { st |= ST_OVERFLOW; return; }
        const unsigned e = cut_poly<double, false>(P, s, um, S[o], S[o], axis_tag(ax));
        freem |= 1u << c;
        c = o;
        if (e) { st |= e; return; }
    }
    for (int i = 0; i < 3; ++i) { S[c].lo[i] = lo[i]; S[c].hi[i] = hi[i]; }
    double mom[10];
    for (;;) {
        Poly<double>& P = S[c];
        bool done_node = true;
        if (P.nv > 0) {
            int dmax = 0, ax = 0;
            for (int i = 0; i < 3; ++i) {
                const int sz = P.hi[i] - P.lo[i];
                if (sz > dmax) { dmax = sz; ax = i; }
            }
            if (dmax <= 1) {
                const unsigned e = reduce_poly(P, mom, 0);
                if (e) { st |= e; return; }
                if (mom[0] > 0.0) {
                    if (P.lo[0] >= a.g.n[0] || P.lo[1] >= a.g.n[1] || P.lo[2] >= a.g.n[2]) {
                        st |= ST_INDEX;
                    } else {
                        const long long gi = ((long long)a.g.n[1] * P.lo[0] + P.lo[1]) * a.g.n[2] + P.lo[2];
                        atomicAdd(&a.m[gi], mass * mom[0]);
                    }
                }
            } else {
                const double coord = a.g.d[ax] * (P.lo[ax] + dmax / 2) + a.g.w0[ax];
                uint32_t um = 0;
                for (int v = 0; v < P.nv; ++v) {
                    s[v] = coord - P.x[v][ax];
                    if (s[v] < 0.0) um |= 1u << v;
                }
                const int nlo = dmax / 2, nup = dmax - dmax / 2;
                if (um == 0) {
                    P.hi[ax] -= nup;
                    done_node = false;
                } else if (um == (1u << P.nv) - 1u) {
                    P.lo[ax] += nlo;
                    done_node = false;
                } else {
                    int l, r;
                    if (!alloc(l) || !alloc(r)) { st |= ST_OVERFLOW; return; }
                    const unsigned e = cut_poly<double, true>(P, s, um, S[l], S[r], axis_tag(ax));
                    if (e) { st |= e; return; }
                    for (int i = 0; i < 3; ++i) {
                        S[l].lo[i] = P.lo[i]; S[l].hi[i] = P.hi[i];
                        S[r].lo[i] = P.lo[i]; S[r].hi[i] = P.hi[i];
                    }
                    S[l].hi[ax] -= nup;
                    S[r].lo[ax] += nlo;
                    freem |= 1u << c;
                    if (top >= NA_NS) { st |= ST_OVERFLOW; return; }
                    stk[top++] = (int8_t)l;
                    c = r;
                    continue;
                }
            }
        }
        if (!done_node) continue;
        freem |= 1u << c;
        if (top == 0) break;
        c = stk[--top];
    }
}

// Pre-pass: flags ST_DEPTH when any tet is too deep for the slot pool, so
// that the deposit kernel, launched next on the same stream, adds nothing.
__global__ void k_noalloc_depth(NaArgs a)
{
    NaState* state = (NaState*)a.scratch;
    bool deep = false;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < a.ntets;
         t += (long long)gridDim.x * blockDim.x) {
        double p[4][3];
        for (int v = 0; v < 4; ++v)
            for (int i = 0; i < 3; ++i) p[v][i] = a.pos[12 * t + 3 * v + i];
        double rb[2][3];
        aabb4(p, rb);
        int lo[3], hi[3];
        index_box(a, rb, lo, hi);
        deep = deep || box_depth(lo, hi) > NA_DMAX;
    }
    if (__any_sync(0xFFFFFFFFu, deep) && (threadIdx.x & 31) == 0) atomicOr(&state->status, ST_DEPTH);
}

__global__ void __launch_bounds__(NA_BLOCK) k_density_noalloc(NaArgs a)
{
    NaState* state = (NaState*)a.scratch;
    if (*(volatile unsigned*)&state->status & ST_DEPTH) return; // the pre-pass rejected the call
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    Poly<double>* S = (Poly<double>*)(a.scratch + NA_STATE + (size_t)tid * NA_REGION);
    const int lane = threadIdx.x & 31;
    unsigned st = 0;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&state->head, 32ull);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= (unsigned long long)a.ntets) break;
        const long long t = (long long)base + lane;
        if (t < a.ntets) deposit_tet(a, t, S, st);
    }
    if (st) atomicOr(&state->status, st);
}

// Device address of the scratch array on the current device.  Looked up on
// every call (cudaGetSymbolAddress allocates nothing), so that it is right
// for the device's current context, also after a cudaDeviceReset.
int noalloc_scratch(unsigned char** out)
{
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        char msg[256];
        snprintf(msg, sizeof(msg), "cudaGetSymbolAddress of the no-alloc scratch failed: %s", cudaGetErrorString(e));
        return report_error(PSIB_ERR_CUDA, msg);
    }
    *out = (unsigned char*)p;
    return PSIB_OK;
}

} // namespace

} // namespace psib

using namespace psib;

extern "C" int psib_voxels_density_noalloc(const psib_grid* grid, const double* tet_pos, const double* tet_mass,
                                           long long ntets, void* stream)
{
    if (!grid || (!tet_pos && ntets > 0)) return report_error(PSIB_ERR_ARG, "grid and tet_pos are required");
    if (ntets < 0) return report_error(PSIB_ERR_ARG, "ntets must not be negative");
    if (!grid->fields[PSIB_M]) return report_error(PSIB_ERR_ARG, "field m is required");
    for (int f = 1; f < 6; ++f)
        if (grid->fields[f])
            return report_error(PSIB_ERR_ARG, "psib_voxels_density_noalloc deposits field m only; pass NULL for the others");
    for (int i = 0; i < 3; ++i) {
        if (grid->n[i] <= 0) return report_error(PSIB_ERR_ARG, "grid n must be positive");
        if (!(grid->d[i] > 0.0)) return report_error(PSIB_ERR_ARG, "grid cell size d must be positive");
    }
    if (ntets == 0) return PSIB_OK;
    if (psib_device_count() <= 0) return report_error(PSIB_ERR_NODEVICE, "no CUDA device is visible");
    unsigned char* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc != PSIB_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    NaArgs a;
    a.pos = tet_pos;
    a.mass = tet_mass;
    a.ntets = ntets;
    for (int i = 0; i < 3; ++i) {
        a.g.n[i] = grid->n[i];
        a.g.w0[i] = grid->window[0][i];
        a.g.w1[i] = grid->window[1][i];
        a.g.d[i] = grid->d[i];
    }
    a.m = grid->fields[PSIB_M];
    a.scratch = scratch;
    // the queue head and the status word start at zero on every call
    cudaError_t e = cudaMemsetAsync(scratch, 0, NA_STATE, st);
    if (e == cudaSuccess) {
        k_noalloc_depth<<<64, 256, 0, st>>>(a);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_density_noalloc<<<NA_THREADS / NA_BLOCK, NA_BLOCK, 0, st>>>(a);
        e = cudaGetLastError();
    }
    NaState h = {};
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, scratch, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        char msg[256];
        snprintf(msg, sizeof(msg), "psib_voxels_density_noalloc: %s", cudaGetErrorString(e));
        return report_error(PSIB_ERR_CUDA, msg);
    }
    if (h.status & ST_DEPTH)
        return report_error(PSIB_ERR_ARG, "a tet is too large for psib_voxels_density_noalloc: the bisection of its "
                                          "voxel index box, sum of ceil(log2(size)) over the axes, is deeper than 12 "
                                          "levels (use psib_voxels); nothing was deposited");
    if (h.status & ST_INDEX) return report_error(PSIB_ERR_INDEX, "voxel index out of range");
    if (h.status) return report_error(PSIB_ERR_OVERFLOW, "a polyhedron outgrew its vertex buffer or slot pool");
    return PSIB_OK;
}
