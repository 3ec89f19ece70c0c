// probe.cu -- this GPU's FMA issue rate, measured: the denominator of the
// FP64 and FP32 rooflines of the clip walk.
//
// Every thread runs eight independent fused multiply-add chains in registers
// (a = a * b + c), so the FP64 (or FP32) pipe is the only bound; the grid fills
// every SM with 1024 threads.  The rate is the best of three timed launches
// after one untimed, 2 flop per FMA.
#include <cuda_runtime.h>

#include "psi_b200.h"

namespace psib {
int report_error(int code, const char* msg);

namespace {

constexpr int PB_BLOCK = 256, PB_BLOCKS_PER_SM = 4, PB_CHAINS = 8;

template <class T>
__global__ void __launch_bounds__(PB_BLOCK) k_fma_chains(T* out, int iters, T b, T c)
{
    T a[PB_CHAINS];
#pragma unroll
    for (int k = 0; k < PB_CHAINS; ++k) a[k] = (T)(threadIdx.x + k) * (T)1e-3;
#pragma unroll 4
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int k = 0; k < PB_CHAINS; ++k) a[k] = fma(a[k], b, c);
    T s = 0;
#pragma unroll
    for (int k = 0; k < PB_CHAINS; ++k) s += a[k];
    out[blockIdx.x * (size_t)blockDim.x + threadIdx.x] = s;
}

template <class T>
int measure(double* tflops)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                 cudaSuccess) {
        cudaGetLastError();
        return report_error(PSIB_ERR_CUDA, "psib_measure_fma_peak: no device attributes");
    }
    const int blocks = sms * PB_BLOCKS_PER_SM;
    const int iters = sizeof(T) == 8 ? 32768 : 65536;
    T* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&out, (size_t)blocks * PB_BLOCK * sizeof(T));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float best = 0.f;
    for (int r = 0; r < 4 && e == cudaSuccess; ++r) {
        e = cudaEventRecord(e0, 0);
        k_fma_chains<T><<<blocks, PB_BLOCK>>>(out, iters, (T)0.9999999, (T)1e-7);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(e1, 0);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (r > 0 && e == cudaSuccess && (best == 0.f || ms < best)) best = ms;
    }
    if (out) cudaFree(out);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess || best <= 0.f) {
        cudaGetLastError();
        return report_error(PSIB_ERR_CUDA, "psib_measure_fma_peak: a CUDA call failed");
    }
    const double flop = 2.0 * PB_CHAINS * (double)iters * blocks * PB_BLOCK;
    *tflops = flop / (best * 1e-3) / 1e12;
    return PSIB_OK;
}

} // namespace
} // namespace psib

extern "C" int psib_measure_fma_peak(int precision, double* tflops)
{
    if (!tflops) return psib::report_error(PSIB_ERR_ARG, "tflops is required");
    if (psib_device_count() <= 0) return psib::report_error(PSIB_ERR_NODEVICE, "no CUDA device is visible");
    if (precision == PSIB_FP64) return psib::measure<double>(tflops);
    if (precision == PSIB_MIXED) return psib::measure<float>(tflops);
    return psib::report_error(PSIB_ERR_ARG, "precision must be PSIB_FP64 (FP64 FMA) or PSIB_MIXED (FP32 FMA)");
}
