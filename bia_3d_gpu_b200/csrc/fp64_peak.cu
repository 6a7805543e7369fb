// fp64_peak.cu -- measured FP64 FMA throughput of the current device.
//
// The pair kernel is bound by the FP64 pipe, so its roofline denominator is the
// sustained DFMA rate of the same GPU.  Every thread runs kChains independent FMA
// chains (enough instruction-level parallelism to cover the DFMA latency), the grid
// fills every SM several times over, and the best of a few timed launches is taken.
#include <cuda_runtime.h>

#include "bia_internal.cuh"

namespace bia {

constexpr int kChains = 8;
constexpr int kPeakThreads = 256;

__global__ void __launch_bounds__(kPeakThreads) fp64_fma_kernel(int iters, double b, double c, double *sink)
{
    double a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; k++) a[k] = (double)(threadIdx.x + k) * 1e-3;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < kChains; k++) a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kChains; k++) s += a[k];
    if (s == 1.2345) sink[blockIdx.x] = s;  // keeps the chains live; never true in practice
}

}  // namespace bia

using namespace bia;

extern "C" int bia_measure_fp64_peak(int device, double *tflops)
{
    if (!tflops) return BIA_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_status(e);
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return cuda_status(e);
    double *sink = nullptr;
    const int blocks = sms * 8;
    e = cudaMalloc(&sink, blocks * sizeof(double));
    if (e != cudaSuccess) return cuda_status(e);
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    const int iters = 1 << 14;
    double best = 0.0;
    for (int rep = 0; rep < 6; rep++) {
        cudaEventRecord(t0);
        fp64_fma_kernel<<<blocks, kPeakThreads>>>(iters, 0.999999, 1e-7, sink);
        cudaEventRecord(t1);
        e = cudaEventSynchronize(t1);
        if (e != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        const double flops = 2.0 * kChains * (double)iters * blocks * kPeakThreads;
        if (rep > 0 && ms > 0.f) best = fmax(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(sink);
    if (e != cudaSuccess) return cuda_status(e);
    *tflops = best;
    return BIA_OK;
}
