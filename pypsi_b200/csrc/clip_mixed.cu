// clip_mixed.cu -- the mixed-precision clip kernels: FP32 plane distances and
// cut-vertex interpolation on tets recentred on their voxel index box; FP64
// window clip and moment sums.  FMA contraction is allowed here.  Both write
// centroid-form records (m0, q-centroid, central q second moment).
#include "psib_clip.cuh"

#include <cstdlib>

namespace psib {

constexpr int DEFAULT_MINB_MIXED = 6;

// Main kernel variants by the minimum number of resident 128-thread blocks
// per SM the register allocation must allow (0: no cap).  More blocks hide more
// scratch latency but force spills; PSIB_CLIP_MINB picks one (default below,
// from measurements at 128^3 -> 256^3).
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_clip_mixed_b(ClipArgs a) { clip_loop<float, NS_MAIN, true>(a); }
__global__ void __launch_bounds__(128) k_clip_mixed(ClipArgs a) { clip_loop<float, NS_MAIN, true>(a); }

static int min_blocks()
{
    const char* v = getenv("PSIB_CLIP_MINB");
    return v && *v ? atoi(v) : DEFAULT_MINB_MIXED;
}

template <class F>
static auto with_variant(F&& f)
{
    switch (min_blocks()) {
    case 4: return f(k_clip_mixed_b<4>);
    case 5: return f(k_clip_mixed_b<5>);
    case 6: return f(k_clip_mixed_b<6>);
    case 8: return f(k_clip_mixed_b<8>);
    default: return f(k_clip_mixed);
    }
}

// PSIB_FP64_CENTRAL: the FP64 walk writing centroid-form records
__global__ void __launch_bounds__(128, 5) k_clip_fp64c(ClipArgs a) { clip_loop<double, NS_MAIN, true>(a); }

// Images with deep trees or long index boxes: FP64 clipping (FP32 would lose
// precision inside a voxel of a long tet), centroid-form records.
__global__ void __launch_bounds__(64) k_clip_mixed_big(ClipArgs a) { clip_loop<double, NS_BIG, true>(a); }

size_t scratch_bytes_mixed(bool big, bool fp64_walk)
{
    return big ? region_bytes<double, NS_BIG>() : fp64_walk ? region_bytes<double, NS_MAIN>() : region_bytes<float, NS_MAIN>();
}

cudaError_t launch_clip_mixed(const ClipArgs& a, bool big, bool fp64_walk, int grid, int block, cudaStream_t s)
{
    if (big) k_clip_mixed_big<<<grid, block, 0, s>>>(a);
    else if (fp64_walk) k_clip_fp64c<<<grid, block, 0, s>>>(a);
    else with_variant([&](auto k) { k<<<grid, block, 0, s>>>(a); return 0; });
    return cudaGetLastError();
}

int clip_blocks_per_sm_mixed(bool big, bool fp64_walk, int block)
{
    int n = 0;
    cudaError_t e = big ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_clip_mixed_big, block, 0)
                    : fp64_walk ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_clip_fp64c, block, 0)
                        : with_variant([&](auto k) { return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, block, 0); });
    if (e != cudaSuccess) { cudaGetLastError(); return 1; }
    return n > 0 ? n : 1;
}

} // namespace psib
