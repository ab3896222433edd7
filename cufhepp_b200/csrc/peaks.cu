// Throughput probe of the FP64 pipe (the roof of the FFNT path), measured on
// the device the engine runs on: every thread runs 8 independent FMA chains.
#include <cuda_runtime.h>

#include "cufhe_b200.h"

namespace {

__global__ void k_dfma(double* sink, int iters, double b, double c)
{
    double a0 = threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3;
    double a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
    for (int i = 0; i < iters; i++) {
        a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
        a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
    }
    const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 0.123456789) sink[threadIdx.x] = s;  // keeps the chains alive
}

}  // namespace

extern "C" int cufhe_measure_fp64_peak(double* tflops)
{
    if (!tflops) return CUFHE_ERR_ARG;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    double* sink = nullptr;
    if (cudaMalloc(&sink, 1024 * sizeof(double)) != cudaSuccess) return CUFHE_ERR_NOMEM;
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_dfma<<<blocks, threads>>>(sink, 256, 0.999999, 1e-9);  // warm-up
    cudaEventRecord(a);
    k_dfma<<<blocks, threads>>>(sink, iters, 0.999999, 1e-9);
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess) return CUFHE_ERR_CUDA;
    *tflops = 2.0 * 8.0 * iters * (double)blocks * threads / (ms * 1e-3) / 1e12;
    return CUFHE_OK;
}
