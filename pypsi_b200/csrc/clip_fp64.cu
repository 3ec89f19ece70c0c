// clip_fp64.cu -- the FP64 clip kernels.  Built with --fmad=false so each
// fragment's moments repeat the reference's double-precision operations
// exactly (see psib_device.cuh).
#include "psib_clip.cuh"

#include <cstdlib>

namespace psib {

// The register-capped main kernel (8 resident blocks) is the default: its
// extra warps hide more scratch latency (measured ~7% faster at 128^3 -> 256^3).
// PSIB_CLIP_OCC=0 selects the 96-register build.
static bool high_occupancy()
{
    const char* v = getenv("PSIB_CLIP_OCC");
    return !(v && v[0] == '0');
}

// images whose bisection tree is at most DMAX_MAIN deep
__global__ void __launch_bounds__(128) k_clip_fp64(ClipArgs a) { clip_loop<double, NS_MAIN, false>(a); }

// the same with registers capped for 8 resident blocks (more warps to hide scratch latency)
__global__ void __launch_bounds__(128, 8) k_clip_fp64_occ(ClipArgs a) { clip_loop<double, NS_MAIN, false>(a); }

// deeper trees
__global__ void __launch_bounds__(64) k_clip_fp64_big(ClipArgs a) { clip_loop<double, NS_BIG, false>(a); }

size_t scratch_bytes_fp64(bool big) { return big ? region_bytes<double, NS_BIG>() : region_bytes<double, NS_MAIN>(); }

cudaError_t launch_clip_fp64(const ClipArgs& a, bool big, int grid, int block, cudaStream_t s)
{
    if (big) k_clip_fp64_big<<<grid, block, 0, s>>>(a);
    else if (high_occupancy()) k_clip_fp64_occ<<<grid, block, 0, s>>>(a);
    else k_clip_fp64<<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

int clip_blocks_per_sm_fp64(bool big, int block)
{
    int n = 0;
    cudaError_t e = big ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_clip_fp64_big, block, 0)
                        : high_occupancy() ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_clip_fp64_occ, block, 0)
                                           : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_clip_fp64, block, 0);
    if (e != cudaSuccess) { cudaGetLastError(); return 1; }
    return n > 0 ? n : 1;
}

} // namespace psib
