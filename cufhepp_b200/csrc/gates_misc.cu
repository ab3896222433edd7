// Elementwise parts of the gate front-end:
//   k_preadd_lvl0   lvl0 pre-add of the BR->IKS order, which the reference
//                   folds into the modulus switch (__BlindRotatePreAdd__,
//                   include/gatebootstrapping_gpu.cuh:1382-1429, :1432-1521)
//   k_finalize_lvl1 lane outputs -> gate outputs of the IKS->BR order
//                   (Mux: + mu, NMux: negate - mu; src/bootstrap_gpu.cu:1557-1672)
//   k_not_copy      Not / Copy (src/bootstrap_gpu.cu:2200-2222)
//   k_copy_rows     wire rows of one shard's wire table into another shard's
//                   table at the same rows (sharded circuits); the
//                   destination may be a peer GPU's memory, written over
//                   NVLink by this device's stores
#include "engine.h"

namespace cufhe {

namespace {

__global__ void k_preadd_lvl0(Plan plan, const uint32_t* __restrict__ in0,
                              const uint32_t* __restrict__ in1, const uint32_t* __restrict__ in2,
                              uint32_t* __restrict__ lane_in)
{
    const int l = blockIdx.x;
    if (l >= plan.lanes) return;
    const LanePreadd p = plan_lane_preadd(plan, l, in0, in1, in2, kTlwe0);
    uint32_t* dst = lane_in + (size_t)l * kTlwe0;
    for (int i = threadIdx.x; i < kTlwe0; i += blockDim.x) {
        uint32_t x = (uint32_t)p.ca * p.a[i];
        if (p.cb) x += (uint32_t)p.cb * p.b[i];
        if (i == kN0) x += p.off;
        dst[i] = x;
    }
}

__global__ void k_finalize_lvl1(Plan plan, const uint32_t* __restrict__ lane_out,
                                uint32_t* __restrict__ out)
{
    const int b = blockIdx.x;
    if (b >= plan.count) return;
    const int op = plan_op(plan, b);
    const int l0 = plan_lane0(plan, b);
    if (l0 < 0) return;
    const LanePreadd p = gate_combine(op, lane_out + (size_t)l0 * kTlwe1,
                                      lane_out + (size_t)(l0 + 1) * kTlwe1);
    uint32_t* dst = out + plan_out_row(plan, b) * kTlwe1;
    for (int i = threadIdx.x; i < kTlwe1; i += blockDim.x) {
        uint32_t x = (uint32_t)p.ca * p.a[i];
        if (p.cb) x += (uint32_t)p.cb * p.b[i];
        if (i == kN) x += p.off;
        dst[i] = x;
    }
}

__global__ void k_not_copy(Plan plan, int words, const uint32_t* __restrict__ in0,
                           uint32_t* __restrict__ out)
{
    const int b = blockIdx.x;
    if (b >= plan.count) return;
    const int op = plan_op(plan, b);
    if (op != kNot && op != kCopy) return;
    const uint32_t* s = in0 + plan_in_row(plan, 0, b) * words;
    uint32_t* d = out + plan_out_row(plan, b) * words;
    for (int i = threadIdx.x; i < words; i += blockDim.x) d[i] = op == kNot ? 0u - s[i] : s[i];
}

// one CTA per listed row; words are 4-byte aligned only (a lvl1 row is 4100 B)
__global__ void k_copy_rows(const int32_t* __restrict__ rows, int nrows, int words,
                            const uint32_t* __restrict__ src, uint32_t* __restrict__ dst)
{
    const int r = blockIdx.x;
    if (r >= nrows) return;
    const size_t base = (size_t)rows[r] * words;
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[base + i] = src[base + i];
}

}  // namespace

cudaError_t launch_copy_rows(const int32_t* rows, int nrows, int words, const uint32_t* src,
                             uint32_t* dst, cudaStream_t st)
{
    if (nrows <= 0) return cudaSuccess;
    k_copy_rows<<<nrows, 256, 0, st>>>(rows, nrows, words, src, dst);
    return cudaGetLastError();
}

cudaError_t launch_preadd_lvl0(const Plan& plan, const uint32_t* in0, const uint32_t* in1,
                               const uint32_t* in2, uint32_t* lane_in, cudaStream_t st)
{
    if (plan.lanes <= 0) return cudaSuccess;
    k_preadd_lvl0<<<plan.lanes, 128, 0, st>>>(plan, in0, in1, in2, lane_in);
    return cudaGetLastError();
}

cudaError_t launch_finalize_lvl1(const Plan& plan, const uint32_t* lane_out, uint32_t* out,
                                 cudaStream_t st)
{
    if (plan.count <= 0) return cudaSuccess;
    k_finalize_lvl1<<<plan.count, 256, 0, st>>>(plan, lane_out, out);
    return cudaGetLastError();
}

cudaError_t launch_not_copy(const Plan& plan, int words, const uint32_t* in0, uint32_t* out,
                            cudaStream_t st)
{
    if (plan.count <= 0) return cudaSuccess;
    k_not_copy<<<plan.count, 256, 0, st>>>(plan, words, in0, out);
    return cudaGetLastError();
}

}  // namespace cufhe
