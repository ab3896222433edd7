// Throughput probes measured on the device the engine runs on:
//  * the FP64 pipe (the roof of the FFNT path): every thread runs 8
//    independent FMA chains;
//  * the INT8 tensor cores (the roof of the exact path): one thread per SM
//    issues back-to-back tcgen05.mma.kind::i8 M128 N256 K32 with random
//    operands (A in TMEM, B in shared memory), the instruction shape of the
//    exact blind rotation's step GEMM.
#include <cuda_runtime.h>

#include "cufhe_b200.h"
#include "tc_util.cuh"

namespace {

using cufhe::desc_kmajor_sw128;
using cufhe::idesc_i8;
using cufhe::mbar_init;
using cufhe::mbar_wait;
using cufhe::smem_u32;
using cufhe::tc_commit;
using cufhe::tc_fence_after;
using cufhe::tc_fence_before;
using cufhe::tc_mma_i8;
using cufhe::tmem_st32;
using cufhe::tmem_wait_st;

// Failure-path probe: one thread waits on an mbarrier that nothing arrives
// at, with `polls` bounded polls (the same bounded-wait pattern as the
// tensor-core kernels, with a short limit), then sets the error flag
// exactly as those kernels do and returns.
__global__ void k_wait_timeout_probe(int* err, uint32_t polls)
{
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    cufhe::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const uint32_t a = smem_u32(&bar);
    bool done = false;
    for (uint32_t i = 0; i < polls && !done; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(0u)
            : "memory");
        done = ok != 0;
    }
    if (!done) atomicOr(err, 4);
}

constexpr int kProbeSmem = 1024 + 32768 + 64;

__global__ void __launch_bounds__(128, 1) k_i8_peak(int iters, int* err)
{
    extern __shared__ __align__(16) unsigned char raw[];
    unsigned char* sm = raw + ((1024u - (smem_u32(raw) & 1023u)) & 1023u);
    uint64_t* done = reinterpret_cast<uint64_t*>(sm + 32768);
    uint32_t* slot = reinterpret_cast<uint32_t*>(done + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < 32768 / 4; i += blockDim.x) {
        uint32_t x = (uint32_t)i * 2654435761u + blockIdx.x * 97u;
        x ^= x >> 15;
        reinterpret_cast<uint32_t*>(sm)[i] = x * 2246822519u;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(slot)), "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    // random A operand: four 32-column slots at column 256, one quadrant per warp
    for (int c = 0; c < 4; c++) {
        uint32_t v[32];
        for (int i = 0; i < 32; i++) {
            uint32_t x = (uint32_t)(lane * 131 + i * 7 + c * 1031 + warp * 65537) * 2654435761u;
            v[i] = (x ^ (x >> 16)) * 2246822519u;
        }
        tmem_st32(tmem + ((uint32_t)(32 * warp) << 16) + 256 + 32 * c, v);
    }
    tmem_wait_st();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0) {
        const uint32_t idesc = idesc_i8(128, 256);
        const uint32_t bbase = smem_u32(sm);
        for (int it = 0; it < iters; it++)
#pragma unroll
            for (int k = 0; k < 4; k++)
                tc_mma_i8(tmem, tmem + 256 + 32 * (it & 3) + 8 * k,
                          desc_kmajor_sw128(bbase + 32 * k), idesc, (it | k) != 0);
        tc_commit(done);
        if (!mbar_wait(done, 0)) atomicOr(err, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

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

extern "C" int cufhe_measure_int8_peak(double* tops)
{
    if (!tops) return CUFHE_ERR_ARG;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int* err = nullptr;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return CUFHE_ERR_NOMEM;
    cudaMemset(err, 0, sizeof(int));
    cudaError_t e = cudaFuncSetAttribute(k_i8_peak, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kProbeSmem);
    const int iters = 1 << 14;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float ms = 0;
    if (e == cudaSuccess) {
        k_i8_peak<<<sms, 128, kProbeSmem>>>(256, err);  // warm-up
        cudaEventRecord(a);
        k_i8_peak<<<sms, 128, kProbeSmem>>>(iters, err);
        cudaEventRecord(b);
        e = cudaEventSynchronize(b);
        cudaEventElapsedTime(&ms, a, b);
    }
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(err);
    if (e != cudaSuccess) return CUFHE_ERR_CUDA;
    if (herr) return CUFHE_ERR_CUDA;  // a bounded wait gave up
    *tops = 2.0 * 128.0 * 256.0 * 32.0 * 4.0 * iters * (double)sms / (ms * 1e-3) / 1e12;
    return CUFHE_OK;
}

namespace cufhe {
cudaError_t launch_wait_timeout_probe(int* err, uint32_t polls, cudaStream_t st)
{
    k_wait_timeout_probe<<<1, 32, 0, st>>>(err, polls);
    return cudaGetLastError();
}
}  // namespace cufhe
