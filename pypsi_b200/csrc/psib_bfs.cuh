// psib_bfs.cuh -- what the breadth-first walks of both precisions share
// (bfs.cu: FP32 positions, bfs_fp64.cu: FP64 positions and q): the queue
// tile layout, warp-wide reservation of queue elements, index boxes, and the
// closing of a cut face whose links are staged in shared memory.
#pragma once
#include "psib_device.cuh"
#include "psib_kernels.h"

namespace psib {

constexpr int BB = 128; // threads per block of every kernel here
constexpr unsigned FULL = 0xFFFFFFFFu;

__device__ __forceinline__ size_t qx(unsigned long long e, int v, int c)
{
    return ((size_t)(e >> 5) * (MAXV * 3) + (size_t)(v * 3 + c)) * 32 + (size_t)(e & 31);
}
__device__ __forceinline__ size_t qn(unsigned long long e, int v)
{
    return ((size_t)(e >> 5) * MAXV + (size_t)v) * 32 + (size_t)(e & 31);
}

// per-thread shared-memory arrays laid out [vertex][thread]
#define AT(arr, v) (arr)[(v) * BB + threadIdx.x]

// Warp-wide exclusive prefix sum of n (every lane calls it); one atomic on
// *count reserves the warp's total.  Returns the warp's first element.
__device__ __forceinline__ unsigned long long warp_reserve(unsigned long long* count, unsigned n, unsigned& off)
{
    const int lane = threadIdx.x & 31;
    unsigned x = n;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    const unsigned total = __shfl_sync(FULL, x, 31);
    off = x - n;
    unsigned long long base = 0;
    if (lane == 0 && total) base = atomicAdd(count, (unsigned long long)total);
    return __shfl_sync(FULL, base, 0);
}

__device__ __forceinline__ void get_box(const PolyQueue& Q, unsigned long long e, int* lo, int* hi)
{
    for (int a = 0; a < 3; ++a) {
        const uint32_t w = Q.box[3 * e + a];
        lo[a] = (int)(w & 0xFFFFu);
        hi[a] = (int)(w >> 16);
    }
}
__device__ __forceinline__ void put_box(const PolyQueue& Q, unsigned long long e, const int* lo, const int* hi)
{
    for (int a = 0; a < 3; ++a) Q.box[3 * e + a] = (uint32_t)lo[a] | ((uint32_t)hi[a] << 16);
}
// the mixed walk's queue element bytes: FP32 positions and links of nv vertices, nv, window mask, box, image
__device__ __forceinline__ unsigned long long elem_bytes(int nv) { return 16ull * nv + 18ull; }

__device__ __forceinline__ bool one_voxel(const int* lo, const int* hi)
{
    return hi[0] - lo[0] <= 1 && hi[1] - lo[1] <= 1 && hi[2] - lo[2] <= 1;
}

// The grid of image t: its cutout's in a batch.
__device__ __forceinline__ const GridDev& grid_of(const ClipArgs& c, long long t)
{
    return c.grids ? c.grids[c.it.grid[t]] : c.g;
}

// Close the cut face of a child whose links are in shared memory (as
// link_cut_vertices does for a polyhedron in memory).
__device__ __forceinline__ bool link_cut_shared(uint32_t* nbs, int base, int nv)
{
    // no return inside the loops: every lane leaves them at the same place, so the warp
    // runs the code after them together
    bool ok = true;
    for (int vs = base; vs < nv && ok; ++vs) {
        int vc = vs, vn = nbget(AT(nbs, vs), 0);
        int steps = 0;
        do {
            if (vn >= nv) {
                ok = false;
                break;
            }
            const uint32_t w = AT(nbs, vn);
            const int k = (nbget(w, 0) == vc) ? 0 : (nbget(w, 1) == vc) ? 1 : (nbget(w, 2) == vc) ? 2 : 3;
            if (k == 3 || ++steps > WALK_CAP) {
                ok = false;
                break;
            }
            vc = vn;
            vn = nbget(AT(nbs, vc), k == 2 ? 0 : k + 1);
        } while (vc < base);
        if (!ok) break;
        AT(nbs, vs) = nbset(AT(nbs, vs), 2, vc);
        AT(nbs, vc) = nbset(AT(nbs, vc), 1, vs);
    }
    return ok;
}

// The edges a cut crosses, (lower vertex vc, link np) as bits 3 vc + np: one new vertex each, so
// a child keeps its side's vertices plus popc of the mask.
__device__ __forceinline__ uint64_t cut_edges(int nv, uint32_t um, const uint32_t* nbI)
{
    uint64_t cm = 0ull;
    for (int vc = 0; vc < nv; ++vc) {
        const uint32_t w = AT(nbI, vc);
        const bool low = !((um >> vc) & 1u);
#pragma unroll
        for (int np = 0; np < 3; ++np)
            if (low && nbget(w, np) < nv && ((um >> nbget(w, np)) & 1u)) cm |= 1ull << (3 * vc + np);
    }
    return cm;
}

} // namespace psib
