// clip_mixed.cu -- the mixed-precision clip-and-deposit kernels: FP32 plane
// distances and cut-vertex interpolation on tets recentred on their voxel
// index box, FP64 window clip, moments, projection and accumulation.  FMA
// contraction is allowed here.
#include "psib_clip.cuh"

namespace psib {

__global__ void __launch_bounds__(128) k_clip_mixed(ClipArgs a)
{
    Poly<float> S[NS_MAIN];
    clip_loop<float, NS_MAIN, false, false>(a, S);
}

__global__ void __launch_bounds__(64) k_clip_mixed_big(ClipArgs a)
{
    Poly<float>* S = (Poly<float>*)a.scratch + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * NS_BIG;
    clip_loop<float, NS_BIG, false, true>(a, S);
}

size_t scratch_bytes_mixed_big() { return sizeof(Poly<float>) * NS_BIG; }

cudaError_t launch_clip_mixed(const ClipArgs& a, bool big, int grid, int block, cudaStream_t s)
{
    if (big) k_clip_mixed_big<<<grid, block, 0, s>>>(a);
    else k_clip_mixed<<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

} // namespace psib
