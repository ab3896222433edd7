// Batched identity key switching lvl1 -> lvl0 (integer, bit-exact).
//
// Semantics of IdentityKeySwitchPreAdd / KeySwitchFromTLWE
// (include/keyswitch_gpu.cuh:13-23, :128-256): x = ca*A + cb*B (+off on b);
// each of the N = 1024 mask coefficients, offset by decompoffset +
// roundoffset, yields t = 7 signed digits v in [-2, 1]; the lvl0 result is
//   res[o] = [o == n0] x_b - sum_{i,j} sign(v) KSK[i][j][|v|-1][o].
//
// The reference runs one CTA per gate in which each thread walks all 1024 x 7
// digits and gathers KSK rows with __ldg (about 4.6 M gather-adds and 13.7 MB
// of KSK bytes per gate).  Here a CTA switches G = 32 gates at once: thread o
// owns output coefficient o of all 32 gates, so each KSK word is loaded once
// (coalesced across o) and applied to 32 gates from registers; the digits of
// all gates are precomputed into shared memory as 14-bit codes.
#include "engine.h"

namespace cufhe {

namespace {

constexpr int kIksGates = 32;
constexpr int kIksThreads = 640;  // >= 637 outputs
constexpr int kT = CUFHE_LVL10_T;
constexpr int kBasebit = CUFHE_LVL10_BASEBIT;

__host__ __device__ constexpr uint32_t iks_offset()
{
    // decompoffset + roundoffset (include/keyswitch_gpu.cuh:13-23, :197-201)
    uint32_t off = 0;
    for (int i = 1; i <= kT; i++) off += 2u << (32 - i * kBasebit);
    return off + (1u << (32 - (1 + kBasebit * kT)));
}

template <int G>
__global__ void __launch_bounds__(kIksThreads) k_iks(int mode, Plan plan, const uint32_t* __restrict__ in0,
                                                     const uint32_t* __restrict__ in1,
                                                     const uint32_t* __restrict__ in2,
                                                     const uint32_t* __restrict__ lane_out,
                                                     const uint32_t* __restrict__ ksk,
                                                     uint32_t* __restrict__ dst)
{
    extern __shared__ __align__(16) unsigned char iks_smem[];
    uint16_t* codes = reinterpret_cast<uint16_t*>(iks_smem);  // [kN][G]
    __shared__ uint32_t xb[G];
    __shared__ LanePreadd pre[G];
    __shared__ int valid[G];

    const int tid = threadIdx.x;
    const int first = blockIdx.x * G;
    const int total = mode == 0 ? plan.lanes : plan.count;

    if (tid < G) {
        const int u = first + tid;
        LanePreadd p = {nullptr, nullptr, 0, 0, 0};
        int ok = 0;
        if (u < total) {
            if (mode == 0) {
                p = plan_lane_preadd(plan, u, in0, in1, in2, kTlwe1);
                ok = 1;
            } else {
                const int op = plan_op(plan, u);
                const int l0 = plan_lane0(plan, u);
                if (l0 >= 0) {
                    p = gate_combine(op, lane_out + (size_t)l0 * kTlwe1,
                                     lane_out + (size_t)(l0 + 1) * kTlwe1);
                    ok = 1;
                }
            }
        }
        pre[tid] = p;
        valid[tid] = ok;
        uint32_t b = 0;
        if (ok) {
            b = (uint32_t)p.ca * p.a[kN] + p.off;
            if (p.cb) b += (uint32_t)p.cb * p.b[kN];
        }
        xb[tid] = b;
    }
    __syncthreads();

    // digit codes: the 14 top bits of x_i + offset hold the 7 two-bit digits
    // (digit j at bits 12-2j, value v = code - 2)
    for (int e = tid; e < kN * G; e += blockDim.x) {
        const int g = e / kN, i = e % kN;
        uint16_t c = 0x2AAA;  // all digits 0 for invalid gates
        if (valid[g]) {
            const LanePreadd& p = pre[g];
            uint32_t x = (uint32_t)p.ca * p.a[i];
            if (p.cb) x += (uint32_t)p.cb * p.b[i];
            c = (uint16_t)((x + iks_offset()) >> (32 - kBasebit * kT));
        }
        codes[i * G + g] = c;
    }
    __syncthreads();

    const int o = tid < kTlwe0 ? tid : kTlwe0 - 1;  // idle threads read in bounds
    uint32_t acc[G];
#pragma unroll
    for (int g = 0; g < G; g++) acc[g] = (o == kN0) ? xb[g] : 0u;

    const uint32_t* kp = ksk + o;
    for (int i = 0; i < kN; i++) {
        uint32_t cw[G / 2];
        const uint4* cp = reinterpret_cast<const uint4*>(codes + i * G);
#pragma unroll
        for (int q = 0; q < G / 8; q++) {
            const uint4 w = cp[q];
            cw[4 * q + 0] = w.x;
            cw[4 * q + 1] = w.y;
            cw[4 * q + 2] = w.z;
            cw[4 * q + 3] = w.w;
        }
        const uint32_t* row = kp + (size_t)i * kT * 2 * kTlwe0;
        uint32_t k1[kT], k2[kT];
#pragma unroll
        for (int j = 0; j < kT; j++) {
            k1[j] = __ldg(row + (2 * j + 0) * kTlwe0);
            k2[j] = __ldg(row + (2 * j + 1) * kTlwe0);
        }
#pragma unroll
        for (int j = 0; j < kT; j++) {
#pragma unroll
            for (int g = 0; g < G; g++) {
                const uint32_t c = (cw[g >> 1] >> ((g & 1) * 16 + 12 - 2 * j)) & 3u;
                // v = c - 2:  -2 -> +KSK[1], -1 -> +KSK[0], 0 -> 0, +1 -> -KSK[0]
                const uint32_t t = (2u - c) * k1[j];
                acc[g] += c == 0 ? k2[j] : t;
            }
        }
    }
    if (tid < kTlwe0) {
#pragma unroll
        for (int g = 0; g < G; g++)
            if (first + g < total && valid[g]) {
                const size_t row = mode == 0 ? (size_t)(first + g) : plan_out_row(plan, first + g);
                dst[row * kTlwe0 + tid] = acc[g];
            }
    }
}

}  // namespace

cudaError_t launch_iks(int mode, const Plan& plan, const uint32_t* in0, const uint32_t* in1,
                       const uint32_t* in2, const uint32_t* lane_out, const uint32_t* ksk,
                       uint32_t* dst, cudaStream_t st)
{
    const int total = mode == 0 ? plan.lanes : plan.count;
    if (total <= 0) return cudaSuccess;
    const int blocks = (total + kIksGates - 1) / kIksGates;
    const size_t smem = sizeof(uint16_t) * kN * kIksGates;
    static DeviceAttrFlags attr;
    const cudaError_t e = set_smem_attr_once(attr, k_iks<kIksGates>, smem);
    if (e != cudaSuccess) return e;
    k_iks<kIksGates><<<blocks, kIksThreads, smem, st>>>(mode, plan, in0, in1, in2, lane_out, ksk,
                                                     dst);
    return cudaGetLastError();
}

}  // namespace cufhe
