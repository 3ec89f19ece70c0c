// clip_fp64.cu -- the FP64 clip-and-deposit kernels.  Built with --fmad=false
// so each fragment's moments repeat the reference's double-precision
// operations exactly (see psib_device.cuh).
#include "psib_clip.cuh"

namespace psib {

template <bool RECORD>
__global__ void __launch_bounds__(128) k_clip_fp64(ClipArgs a)
{
    Poly<double> S[NS_MAIN];
    clip_loop<double, NS_MAIN, RECORD, false>(a, S);
}

// Tet images whose bisection tree is deeper than DMAX_MAIN: slots in a global
// scratch buffer, NS_BIG per thread.
template <bool RECORD>
__global__ void __launch_bounds__(64) k_clip_fp64_big(ClipArgs a)
{
    Poly<double>* S = (Poly<double>*)a.scratch + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * NS_BIG;
    clip_loop<double, NS_BIG, RECORD, true>(a, S);
}

size_t scratch_bytes_fp64_big() { return sizeof(Poly<double>) * NS_BIG; }

cudaError_t launch_clip_fp64(const ClipArgs& a, bool big, bool record, int grid, int block, cudaStream_t s)
{
    if (big) {
        if (record) k_clip_fp64_big<true><<<grid, block, 0, s>>>(a);
        else k_clip_fp64_big<false><<<grid, block, 0, s>>>(a);
    } else {
        if (record) k_clip_fp64<true><<<grid, block, 0, s>>>(a);
        else k_clip_fp64<false><<<grid, block, 0, s>>>(a);
    }
    return cudaGetLastError();
}

} // namespace psib
