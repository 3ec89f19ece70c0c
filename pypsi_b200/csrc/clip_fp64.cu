// clip_fp64.cu -- the FP64 clip kernels.  Built with --fmad=false so each
// fragment's moments repeat the reference's double-precision operations
// exactly (see psib_device.cuh).
#include "psib_clip.cuh"

#include <cstdlib>

namespace psib {

constexpr int DEFAULT_MINB_FP64 = 6;

// Main kernel variants by the minimum number of resident 128-thread blocks
// per SM the register allocation must allow (0: no cap); PSIB_CLIP_MINB picks
// one (default below, from measurements at 128^3 -> 256^3).
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_clip_fp64_b(ClipArgs a) { clip_loop<double, NS_MAIN, false>(a); }
__global__ void __launch_bounds__(128) k_clip_fp64(ClipArgs a) { clip_loop<double, NS_MAIN, false>(a); }

static int min_blocks()
{
    const char* v = getenv("PSIB_CLIP_MINB");
    return v && *v ? atoi(v) : DEFAULT_MINB_FP64;
}

template <class F>
static auto with_variant(F&& f)
{
    switch (min_blocks()) {
    case 4: return f(k_clip_fp64_b<4>);
    case 5: return f(k_clip_fp64_b<5>);
    case 6: return f(k_clip_fp64_b<6>);
    case 8: return f(k_clip_fp64_b<8>);
    default: return f(k_clip_fp64);
    }
}

// deeper trees
__global__ void __launch_bounds__(64) k_clip_fp64_big(ClipArgs a) { clip_loop<double, NS_BIG, false>(a); }

// adjoint of the density deposit: the FP64 walk again, pulling dL/dm back to the particles
__global__ void __launch_bounds__(128, 4) k_adjoint(ClipArgs a) { clip_loop<double, NS_MAIN, false, true>(a); }
__global__ void __launch_bounds__(64) k_adjoint_big(ClipArgs a) { clip_loop<double, NS_BIG, false, true>(a); }

// the adjoint of every field (adj_coef set): positions, velocities and masses
__global__ void __launch_bounds__(128) k_adjoint_full(ClipArgs a) { clip_loop<double, NS_MAIN, false, true, true>(a); }
__global__ void __launch_bounds__(64) k_adjoint_full_big(ClipArgs a)
{
    clip_loop<double, NS_BIG, false, true, true>(a);
}

cudaError_t launch_adjoint(const ClipArgs& a, bool big, int grid, int block, cudaStream_t s)
{
    if (a.adj_coef) {
        if (big) k_adjoint_full_big<<<grid, block, 0, s>>>(a);
        else k_adjoint_full<<<grid, block, 0, s>>>(a);
    } else if (big) {
        k_adjoint_big<<<grid, block, 0, s>>>(a);
    } else {
        k_adjoint<<<grid, block, 0, s>>>(a);
    }
    return cudaGetLastError();
}

int adjoint_blocks_per_sm(bool big, int block, bool full)
{
    int n = 0;
    cudaError_t e;
    if (full)
        e = big ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adjoint_full_big, block, 0)
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adjoint_full, block, 0);
    else
        e = big ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adjoint_big, block, 0)
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adjoint, block, 0);
    if (e != cudaSuccess) { cudaGetLastError(); return 1; }
    return n > 0 ? n : 1;
}

size_t scratch_bytes_fp64(bool big) { return big ? region_bytes<double, NS_BIG>() : region_bytes<double, NS_MAIN>(); }

cudaError_t launch_clip_fp64(const ClipArgs& a, bool big, int grid, int block, cudaStream_t s)
{
    if (big) k_clip_fp64_big<<<grid, block, 0, s>>>(a);
    else with_variant([&](auto k) { k<<<grid, block, 0, s>>>(a); return 0; });
    return cudaGetLastError();
}

int clip_blocks_per_sm_fp64(bool big, int block)
{
    int n = 0;
    cudaError_t e = big ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_clip_fp64_big, block, 0)
                        : with_variant([&](auto k) { return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, block, 0); });
    if (e != cudaSuccess) { cudaGetLastError(); return 1; }
    return n > 0 ? n : 1;
}

} // namespace psib
