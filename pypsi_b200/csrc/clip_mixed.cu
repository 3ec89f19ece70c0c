// clip_mixed.cu -- the mixed-precision clip kernels: FP32 plane distances and
// cut-vertex interpolation on tets recentred on their voxel index box; FP64
// window clip and moment sums.  FMA contraction is allowed here.  Both write
// centroid-form records (m0, q-centroid, central q second moment).
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

__global__ void __launch_bounds__(128) k_clip_mixed(ClipArgs a) { clip_loop<float, NS_MAIN, true>(a); }

// the same with registers capped for 8 resident blocks (more warps to hide scratch latency)
__global__ void __launch_bounds__(128, 8) k_clip_mixed_occ(ClipArgs a) { clip_loop<float, NS_MAIN, true>(a); }

// Images with deep trees or long index boxes: FP64 clipping (FP32 would lose
// precision inside a voxel of a long tet), centroid-form records.
__global__ void __launch_bounds__(64) k_clip_mixed_big(ClipArgs a) { clip_loop<double, NS_BIG, true>(a); }

size_t scratch_bytes_mixed(bool big) { return big ? region_bytes<double, NS_BIG>() : region_bytes<float, NS_MAIN>(); }

cudaError_t launch_clip_mixed(const ClipArgs& a, bool big, int grid, int block, cudaStream_t s)
{
    if (big) k_clip_mixed_big<<<grid, block, 0, s>>>(a);
    else if (high_occupancy()) k_clip_mixed_occ<<<grid, block, 0, s>>>(a);
    else k_clip_mixed<<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

int clip_blocks_per_sm_mixed(bool big, int block)
{
    int n = 0;
    cudaError_t e = big ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_clip_mixed_big, block, 0)
                        : high_occupancy() ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_clip_mixed_occ, block, 0)
                                           : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_clip_mixed, block, 0);
    if (e != cudaSuccess) { cudaGetLastError(); return 1; }
    return n > 0 ? n : 1;
}

} // namespace psib
