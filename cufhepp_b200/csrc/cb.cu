// CMUX and CMUX lookup tables (the private key switching of circuit
// bootstrapping runs on the tensor cores, iks_tc.cu).
//
//   k_cmux     CMUX d0 + ExtProd(C, d1 - d0) with a Fourier-domain TRGSW<lvl1>
//              of L digits of BGBIT bits (the reference's CMUX,
//              src/bootstrap_gpu.cu:704-813, with its lvl1 gadget l = 2,
//              Bgbit = 8, or the circuit-bootstrapping gadget l = 3, Bgbit = 6).
//   k_lut_leaves / k_extract8
//              leaves and outputs of 8-bit -> 8-bit lookup tables evaluated as
//              CMUX trees with the 8 output bits packed in coefficients 0..7.

#include "cufhe_b200.h"
#include "engine.h"
#include "fft64.cuh"

namespace cufhe {

namespace {


// signed digit d (0 = most significant) of an offset Torus32 value, BGBIT bits
template <int L, int BGBIT>
__device__ __forceinline__ double gadget_digit(uint32_t t, int d)
{
    return (double)((int32_t)((t >> (32 - (d + 1) * BGBIT)) & ((1u << BGBIT) - 1)) -
                    (int32_t)(1u << (BGBIT - 1)));
}

template <int L, int BGBIT>
constexpr uint32_t gadget_offset()
{
    uint32_t off = 0;
    for (int i = 1; i <= L; i++) off += (1u << (BGBIT - 1)) << (32 - i * BGBIT);
    return off + (1u << (32 - L * BGBIT - 1));
}

// One CMUX per CTA, 2L warps: warp r = (input poly j, digit d) transforms its
// digit row; thread f (bin) multiplies-accumulates with the key; warps 0, 1
// transform back and add d0.
template <int L, int BGBIT>
__global__ void __launch_bounds__(64 * L) k_cmux(CmuxPlan p, const double2* __restrict__ psi,
                                                 const double2* __restrict__ tw512)
{
    extern __shared__ __align__(16) unsigned char cmux_smem[];
    double2 (*slots)[kSlotStride] = reinterpret_cast<double2 (*)[kSlotStride]>(cmux_smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x;
    const int g = c / p.per, m = c % p.per;
    const size_t node = (size_t)g * p.node_stride_g + (size_t)m * p.node_stride_m;
    const uint32_t* d0 = p.d0 + node * kTrlwe;
    const uint32_t* d1 = p.d1 + node * kTrlwe;
    const double2* key = p.trgsw + (size_t)g * p.trgsw_stride;
    uint32_t* out = p.out + ((size_t)g * p.per + m) * kTrlwe;
    constexpr uint32_t kOffG = gadget_offset<L, BGBIT>();
    {
        const int j = warp / L, d = warp % L;
        double2 v[16];
#pragma unroll
        for (int n2 = 0; n2 < 16; n2++) {
            const int n = lane + 32 * n2;
            const uint32_t lo = d1[j * kN + n] - d0[j * kN + n];
            const uint32_t hi = d1[j * kN + n + kHalfN] - d0[j * kN + n + kHalfN];
            const double2 z = make_double2(gadget_digit<L, BGBIT>(lo + kOffG, d),
                                           gadget_digit<L, BGBIT>(hi + kOffG, d));
            v[n2] = cmul(z, __ldg(&psi[n]));
        }
        fft512_warp<1>(v, slots[warp], tw512, lane);
#pragma unroll
        for (int mm = 0; mm < 16; mm++) slots[warp][(lane & 15) + 16 * mm + 256 * (lane >> 4)] = v[mm];
    }
    __syncthreads();
    for (int f = threadIdx.x; f < kHalfN; f += blockDim.x) {
        double2 o0 = make_double2(0.0, 0.0), o1 = o0;
#pragma unroll
        for (int r = 0; r < 2 * L; r++) {
            const double2 z = slots[r][f];
            o0 = cfma(o0, z, __ldg(&key[(r * 2 + 0) * kHalfN + f]));
            o1 = cfma(o1, z, __ldg(&key[(r * 2 + 1) * kHalfN + f]));
        }
        slots[0][f] = o0;  // only this thread reads or writes bin f
        slots[1][f] = o1;
    }
    __syncthreads();
    if (warp < 2) {
        const int oj = warp;
        double2 v[16];
#pragma unroll
        for (int n2 = 0; n2 < 16; n2++) v[n2] = slots[oj][lane + 32 * n2];
        __syncwarp();
        fft512_warp<-1>(v, slots[oj], tw512, lane);
#pragma unroll
        for (int mm = 0; mm < 16; mm++) {
            const int n = (lane & 15) + 16 * mm + 256 * (lane >> 4);
            // untwist conj(psi^n), / 512, x 2^32 => x 2^23; llrint as the reference
            const double2 u = cmulc(v[mm], __ldg(&psi[n]));
            const uint32_t lo = (uint32_t)__double2ll_rn(u.x * 0x1p23);
            const uint32_t hi = (uint32_t)__double2ll_rn(u.y * 0x1p23);
            out[oj * kN + n] = d0[oj * kN + n] + lo;
            out[oj * kN + n + kHalfN] = d0[oj * kN + n + kHalfN] + hi;
        }
    }
}

// leaves of q lookup tables: node (q, x) = (0, sum_b (bit b of lut[x] ? mu : -mu) X^b)
__global__ void k_lut_leaves(const uint8_t* __restrict__ luts, int q, uint32_t mu,
                             uint32_t* __restrict__ nodes)
{
    const size_t node = blockIdx.x;  // q * 256 + x
    if (node >= (size_t)q * 256) return;
    const uint8_t v = luts[node];
    uint32_t* t = nodes + node * kTrlwe;
    for (int i = threadIdx.x; i < kTrlwe; i += blockDim.x) {
        uint32_t w = 0;
        if (i >= kN && i < kN + 8) w = ((v >> (i - kN)) & 1) ? mu : 0u - mu;
        t[i] = w;
    }
}

// SampleExtract at coefficients 0..7 of each root TRLWE -> TLWE<lvl1> [q][8][1025]
__global__ void k_extract8(const uint32_t* __restrict__ roots, int q, uint32_t* __restrict__ out)
{
    const int idx = blockIdx.x;  // q * 8 + b
    if (idx >= q * 8) return;
    const int b = idx & 7;
    const uint32_t* acc = roots + (size_t)(idx >> 3) * kTrlwe;
    uint32_t* o = out + (size_t)idx * kTlwe1;
    for (int n = threadIdx.x; n <= kN; n += blockDim.x)
        o[n] = n == kN ? acc[kN + b] : (n <= b ? acc[b - n] : 0u - acc[kN + b - n]);
}

}  // namespace

// The FFT constants of this translation unit (fft64.cuh keeps them per file)
cudaError_t upload_cb_constants(void)
{
    double2 w[16];
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < 16; k++) {
        const long double a = 2 * pi * k / 32;
        w[k] = make_double2((double)cosl(a), (double)sinl(a));
    }
    return cudaMemcpyToSymbol(c_w32, w, sizeof(w));
}

template <int L, int BGBIT>
static cudaError_t launch_cmux_t(const CmuxPlan& p, const Fp64Tables& t, cudaStream_t st)
{
    constexpr size_t smem = sizeof(double2) * 2 * L * kSlotStride;
    static DeviceAttrFlags attr;
    {
        const cudaError_t e = set_smem_attr_once(attr, k_cmux<L, BGBIT>, smem);
        if (e != cudaSuccess) return e;
    }
    k_cmux<L, BGBIT><<<p.count, 64 * L, smem, st>>>(p, t.psi, t.tw512);
    return cudaGetLastError();
}

cudaError_t launch_cmux(int gadget, const CmuxPlan& p, const Fp64Tables& t, cudaStream_t st)
{
    if (p.count <= 0) return cudaSuccess;
    return gadget == CUFHE_GADGET_CB ? launch_cmux_t<3, 6>(p, t, st) : launch_cmux_t<2, 8>(p, t, st);
}

cudaError_t launch_lut_leaves(const uint8_t* luts, int q, uint32_t mu, uint32_t* nodes,
                              cudaStream_t st)
{
    if (q <= 0) return cudaSuccess;
    k_lut_leaves<<<q * 256, 256, 0, st>>>(luts, q, mu, nodes);
    return cudaGetLastError();
}

cudaError_t launch_extract8(const uint32_t* roots, int q, uint32_t* out, cudaStream_t st)
{
    if (q <= 0) return cudaSuccess;
    k_extract8<<<q * 8, 256, 0, st>>>(roots, q, out);
    return cudaGetLastError();
}

}  // namespace cufhe
