// lvl0 -> lvl2 FP64 FFNT blind rotation (N = 2048, k = 1, l = 4, Bgbit = 10,
// Torus64) with fused SampleExtract: the lvl02param instantiation of
// __BlindRotate__ / __BlindRotateKeyBundle__ (include/gatebootstrapping_gpu.cuh
// :801-884, :895-1033) that the *_lvl02 gates run (src/cufhe_gates_gpu.cu
// :826-979).
//   bar = 2N - (b >> 20), abar_i = (a_i + 2^19) >> 20   (N = 2048)
//   digits: 4 signed 10-bit digits of t + offset, offset = sum 512 2^{64-10i}
//           + 2^23 (rounding), include/gatebootstrapping_gpu.cuh:20-29
//   inverse: round to Torus64 by the mantissa-shift conversion of
//            include/utils_gpu.cuh:48-65 (truncating, wraps mod 2^64)
//
// B200 layout.  The 1024-point FFNT is split into two 512-point halves over
// the even and odd folded samples, each one warp transform (fft64.cuh); the
// radix-2 step that joins them (Z[k] = E[k] +- psi2^{4k} O[k]) is fused into
// the key multiply-accumulate, and its inverse (E' = Z[k] + Z[k+512],
// O' = (Z[k] - Z[k+512]) psi2^{-4k}) into the MAC's epilogue.  A CTA carries
// G lanes; per step the eight digit rows are processed in two chunks of four
// (the rows of input polynomial a, then b) so that the spectra of one lane
// fit 67 KB of shared memory:
//   F  warp (g, d, parity): digits, fold, twist, 512-point FFT -> slot
//   M  thread (bin pair, lane): radix-2 join, key MAC into registers
//      (after the second chunk: inverse radix-2 split -> slots)
//   I  warp (g, j, parity): inverse 512-point FFT, untwist, Torus64 rounding
// Batches of up to one lane per SM pair run k_br2_fp64_clu instead: one lane per
// cluster of two CTAs on two SMs, the key MAC split between them and the
// products gathered through distributed shared memory.
// The root table psi2^s (psi2 = e^{i pi / 2048}) keeps s in [0, 512] only
// (8 KB); other powers follow from psi2^{1024} = i and
// psi2^{1024 - s} = i conj(psi2^s).
#include <cooperative_groups.h>

#include "engine.h"
#include "fft64.cuh"

namespace cufhe {

namespace {

constexpr int kN2 = CUFHE_LVL2_N;          // 2048
constexpr int kTlwe2 = CUFHE_TLWE2_WORDS;  // 2049
constexpr int kTrlwe2 = CUFHE_TRLWE2_WORDS;  // 4096
constexpr int kAbarStride2 = 640;
constexpr uint64_t kDecOffset2 = (512ull << 54) + (512ull << 44) + (512ull << 34) +
                                 (512ull << 24) + (1ull << 23);
constexpr size_t kTrgswF2 = 8 * 2 * 1024;  // double2 per Fourier TRGSW<lvl2>

template <int G>
constexpr size_t br2_smem_bytes()
{
    return sizeof(double2) * G * 8 * kSlotStride + sizeof(double2) * kPsi2Entries +
           sizeof(uint64_t) * G * kTrlwe2 + sizeof(uint16_t) * G * kAbarStride2;
}

// shared memory requested per CTA: more than half an SM, so that every CTA
// has an SM (and its whole register file) to itself
constexpr size_t kSmemOneCta = 120 * 1024;

// Shared-memory position of psi2^s (s in [0, 512]): the low 3 bits XORed
// with the next 3, so that the kernels' strided gathers (psi2^{(1+4k) a},
// psi2^{4 k}, psi2^{2 lane + p}, psi2^{8 lane}) spread over the banks: 2.3
// wavefronts per 8 lanes on average for the KeyBundle roots (4.6 in natural
// order), 1 to 1.5 for the others (2 to 8).
__device__ __forceinline__ uint32_t psi2_pos(uint32_t s) { return s ^ ((s >> 3) & 7u); }

// psi2^t for any t (mod 4096) from the table of s in [0, 512] (kSwz: the
// shared-memory copy, in psi2_pos order; else the natural-order table)
template <bool kSwz = true>
__device__ __forceinline__ double2 psi2_at(const double2* tab, uint32_t t)
{
    const uint32_t q = (t >> 10) & 3u;
    const uint32_t s = t & 1023u;
    const bool refl = s > 512u;
    const uint32_t i = refl ? 1024u - s : s;
    const double2 w = tab[kSwz ? psi2_pos(i) : i];
    double2 v = refl ? make_double2(w.y, w.x) : w;
    if (q & 1u) v = make_double2(-v.y, v.x);
    if (q & 2u) v = make_double2(-v.x, -v.y);
    return v;
}

// i^m v (exact: swaps and negations, as in psi2_at), so that
// psi2_at(t + 1024 m) = mul_ipow(psi2_at(t), m)
__device__ __forceinline__ double2 mul_ipow(double2 v, uint32_t m)
{
    if (m & 1u) v = make_double2(-v.y, v.x);
    if (m & 2u) v = make_double2(-v.x, -v.y);
    return v;
}

__device__ __forceinline__ double digit2_of(uint64_t t, int d)
{
    return (double)((int32_t)((t >> (54 - 10 * d)) & 1023u) - 512);
}

// Torus64 value of x (already scaled by 2^64): mantissa shift, truncating,
// modulo 2^64
__device__ __forceinline__ uint64_t to_torus64(double x)
{
    const uint64_t i = (uint64_t)__double_as_longlong(x);
    const int expo = (int)((i >> 52) & 0x7FF);
    const uint64_t m = (i & 0x000FFFFFFFFFFFFFull) | 0x0010000000000000ull;
    const int shift = expo - 1075;
    uint64_t v = 0;
    if (shift >= 0 && shift < 64)
        v = m << shift;
    else if (shift < 0 && shift > -64)
        v = m >> (-shift);
    if (expo == 0) v = 0;
    return (i >> 63) ? 0ull - v : v;
}

// One CTA per SM (launch bound 1, and at least 120 KB of shared memory
// requested): the transforms and the MAC want more than the 128 registers per
// thread that two CTAs per SM would leave (2048 lanes 70.1 -> 66.2 ms, 148
// lanes 9.2 -> 4.7 ms against two one-lane CTAs per SM).
template <bool KB, int G>
__global__ void __launch_bounds__(G * 256, 1)
    k_br2_fp64(const uint32_t* __restrict__ lane_in, int lanes, uint64_t mu,
               const double2* __restrict__ bkf, const double2* __restrict__ psi2, int steps,
               uint64_t* __restrict__ acc_out, uint64_t* __restrict__ lane_out, int in_count,
               int mu_shift)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double2* spec = reinterpret_cast<double2*>(smem);       // [G][8][kSlotStride]
    double2* tab = spec + G * 8 * kSlotStride;              // [kPsi2Entries]
    uint64_t* acc = reinterpret_cast<uint64_t*>(tab + kPsi2Entries);  // [G][2][2048]
    uint16_t* abar = reinterpret_cast<uint16_t*>(acc + G * kTrlwe2);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int lane_base = blockIdx.x * G;

    for (int t = tid; t < kPsi2Entries; t += blockDim.x) tab[psi2_pos(t)] = psi2[t];
#pragma unroll 1
    for (int g = 0; g < G; g++) {
        const int l = lane_base + g;
        const bool ok = l < lanes;
        // lane l rotates input l mod in_count with test value mu >> (mu_shift
        // (l div in_count)): several test polynomials over one input batch
        const int src = ok ? l % in_count : 0;
        const uint64_t mul = mu >> (mu_shift * (ok ? l / in_count : 0));
        const uint32_t* x = lane_in + (size_t)src * kTlwe0;
        for (int i = tid; i < kN0; i += blockDim.x)
            abar[g * kAbarStride2 + i] = ok ? (uint16_t)((x[i] + (1u << 19)) >> 20) : 0;
        const uint32_t bar = ok ? 2u * kN2 - (x[kN0] >> 20) : 2u * kN2;
        for (int i = tid; i < kN2; i += blockDim.x) {
            acc[g * kTrlwe2 + i] = 0;
            uint64_t v;
            if (bar == 2u * kN2)
                v = mul;
            else
                v = (((uint32_t)i < (bar & (kN2 - 1))) ^ (bar >> 11)) ? 0ull - mul : mul;
            acc[g * kTrlwe2 + kN2 + i] = v;
        }
    }
    __syncthreads();

    const int total = KB ? kN0 / 2 : kN0;
    const int nsteps = (steps < 0 || steps > total) ? total : steps;

#pragma unroll 1
    for (int p = 0; p < nsteps; p++) {
        // MAC accumulators: [combo][j][bin half]; combo = (pair index, lane)
        double2 out[2][2][2];
        const double2* bk = bkf + (size_t)p * (KB ? 3 : 1) * kTrgswF2;
#pragma unroll 1
        for (int c = 0; c < 2; c++) {
            // ---- F: digits of input polynomial c, row d, parity par
            {
                const int g = warp >> 3, s = warp & 7, d = s >> 1, par = s & 1;
                const uint64_t* a = acc + g * kTrlwe2 + c * kN2;
                const uint32_t ab = KB ? 0u : abar[g * kAbarStride2 + p];
                const uint32_t abm = ab & (kN2 - 1), abn = ab >> 11;
                double2 v[16];
#pragma unroll
                for (int n2 = 0; n2 < 16; n2++) {
                    const int n = 2 * (lane + 32 * n2) + par;
                    uint64_t lo = a[n], hi = a[n + 1024];
                    if constexpr (!KB) {
                        // X^abar acc - acc (include/gatebootstrapping_gpu.cuh:114-138)
                        uint64_t rl = a[(n - ab) & (kN2 - 1)];
                        uint64_t rh = a[(n + 1024 - ab) & (kN2 - 1)];
                        rl = (((uint32_t)n < abm) ^ abn) ? 0ull - rl : rl;
                        rh = (((uint32_t)(n + 1024) < abm) ^ abn) ? 0ull - rh : rh;
                        lo = rl - lo;
                        hi = rh - hi;
                    }
                    v[n2] = make_double2(digit2_of(lo + kDecOffset2, d),
                                         digit2_of(hi + kDecOffset2, d));
                    if (n2) v[n2] = cmul(v[n2], c_tw32[n2]);
                }
                double2* slot = spec + (g * 8 + s) * kSlotStride;
                dft512_fwd_post(v, slot, lane, psi2_at(tab, 2u * lane + par),
                                psi2_at(tab, 8u * lane));
#pragma unroll
                for (int q = 0; q < 16; q++) slot[ffnt_pos(lane, q)] = v[q];
            }
            __syncthreads();

            // ---- M: radix-2 join + key multiply-accumulate
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int k = G == 1 ? tid + 256 * q : tid;  // bin pair (k, k + 512)
                const int g = G == 1 ? 0 : q;
                const double2 w4 = psi2_at(tab, 4u * (uint32_t)k);
                const double2* sl = spec + g * 8 * kSlotStride;
                double2 fac[2][3];
                if (KB) {
                    // bin k + 512: the roots of bin k times i^{2 a} (exact)
                    const uint32_t a0 = abar[g * kAbarStride2 + 2 * p];
                    const uint32_t a1 = abar[g * kAbarStride2 + 2 * p + 1];
                    const uint32_t am[3] = {a0 + a1, a0, a1};
                    const uint32_t e = 1u + 4u * (uint32_t)k;
#pragma unroll
                    for (int f = 0; f < 3; f++) {
                        fac[0][f] = psi2_at(tab, e * am[f]);
                        fac[1][f] = mul_ipow(fac[0][f], 2u * am[f]);
                    }
#pragma unroll
                    for (int h = 0; h < 2; h++)
#pragma unroll
                        for (int f = 0; f < 3; f++) fac[h][f].x -= 1.0;
                }
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int bin = k + 512 * h;
                    double2 Z[4];
#pragma unroll
                    for (int d = 0; d < 4; d++) {
                        const double2 E = sl[(2 * d) * kSlotStride + k];
                        const double2 wo = cmul(sl[(2 * d + 1) * kSlotStride + k], w4);
                        Z[d] = h ? csub(E, wo) : cadd(E, wo);
                    }
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        double2 o = c ? out[q][j][h] : make_double2(0.0, 0.0);
                        if (KB) {
                            double2 s0 = make_double2(0.0, 0.0), s1 = s0, s2 = s0;
#pragma unroll
                            for (int d = 0; d < 4; d++) {
                                const int r = c * 4 + d;
                                const size_t ki = ((size_t)r * 2 + j) * 1024 + bin;
                                s0 = cfma(s0, Z[d], __ldg(&bk[0 * kTrgswF2 + ki]));
                                s1 = cfma(s1, Z[d], __ldg(&bk[1 * kTrgswF2 + ki]));
                                s2 = cfma(s2, Z[d], __ldg(&bk[2 * kTrgswF2 + ki]));
                            }
                            if (j == c) {
                                // FFNT(H) of row (c, d) = 2^{-10 (d + 1)}
#pragma unroll
                                for (int d = 0; d < 4; d++) {
                                    const double sc = d == 0 ? 0x1p-10 : d == 1 ? 0x1p-20
                                                    : d == 2 ? 0x1p-30 : 0x1p-40;
                                    o.x = fma(Z[d].x, sc, o.x);
                                    o.y = fma(Z[d].y, sc, o.y);
                                }
                            }
                            o = cfma(o, fac[h][0], s0);
                            o = cfma(o, fac[h][1], s1);
                            o = cfma(o, fac[h][2], s2);
                        } else {
#pragma unroll
                            for (int d = 0; d < 4; d++) {
                                const int r = c * 4 + d;
                                o = cfma(o, Z[d], __ldg(&bk[((size_t)r * 2 + j) * 1024 + bin]));
                            }
                        }
                        out[q][j][h] = o;
                    }
                }
                if (c == 1) {
                    // inverse radix-2 split into slots (j, parity) of this lane;
                    // only this thread touches bin k of these slots
                    double2* so = spec + g * 8 * kSlotStride;
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        so[(2 * j) * kSlotStride + k] = cadd(out[q][j][0], out[q][j][1]);
                        so[(2 * j + 1) * kSlotStride + k] =
                            cmulc(csub(out[q][j][0], out[q][j][1]), w4);
                    }
                }
            }
            __syncthreads();
        }

        // ---- I: inverse 512-point FFT, untwist, round, warp (g, j, parity)
        if (warp < 4 * G) {
            const int g = warp >> 2, j = (warp >> 1) & 1, par = warp & 1;
            double2* slot = spec + (g * 8 + 2 * j + par) * kSlotStride;
            double2 v[16];
#pragma unroll
            for (int n2 = 0; n2 < 16; n2++) v[n2] = slot[lane + 32 * n2];
            __syncwarp();
            dft512_inv_raw(v, slot, lane, psi2_at(tab, 8u * lane));
            const int k2 = lane & 15, hh = lane >> 4;
            const double2 u = psi2_at(tab, 2u * (uint32_t)(k2 + 128 * hh) + par);
            uint64_t* a = acc + g * kTrlwe2 + j * kN2;
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int n = 2 * ffnt_pos(lane, q) + par;
                // untwisted value / 1024, then x 2^64  =>  x 2^54 (in c_utwq)
                const double2 z = cmul(cmulc(v[q], u), c_utwq[q]);
                const uint64_t lo = to_torus64(z.x);
                const uint64_t hi = to_torus64(z.y);
                if (KB) {
                    a[n] = lo;
                    a[n + 1024] = hi;
                } else {
                    a[n] += lo;
                    a[n + 1024] += hi;
                }
            }
        }
        __syncthreads();
    }

    // ---- epilogue: accumulator and/or SampleExtract (index 0)
    for (int g = 0; g < G; g++) {
        const int l = lane_base + g;
        if (l >= lanes) break;
        const uint64_t* a = acc + g * kTrlwe2;
        if (acc_out)
            for (int i = tid; i < kTrlwe2; i += blockDim.x) acc_out[(size_t)l * kTrlwe2 + i] = a[i];
        if (lane_out) {
            uint64_t* o = lane_out + (size_t)l * kTlwe2;
            for (int i = tid; i <= kN2; i += blockDim.x)
                o[i] = i == kN2 ? a[kN2] : (i == 0 ? a[0] : 0ull - a[kN2 - i]);
        }
    }
}

// BK<lvl2> polynomial -> Fourier domain, natural bin order: signed int64
// scaled by 2^-64, fold, twist, 1024-point FFT as two halves joined by one
// radix-2 step (src/bootstrap_gpu.cu:59-112 at lvl2param).  One CTA of two
// warps per polynomial.
__global__ void __launch_bounds__(64) k_bk2_to_fft(const uint64_t* __restrict__ bk, int npolys,
                                                  const double2* __restrict__ psi2,
                                                  double2* __restrict__ out)
{
    __shared__ __align__(16) double2 slots[2][kSlotStride];
    const int par = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int poly = blockIdx.x;
    if (poly >= npolys) return;
    const uint64_t* src = bk + (size_t)poly * kN2;
    double2 v[16];
#pragma unroll
    for (int n2 = 0; n2 < 16; n2++) {
        const int n = 2 * (lane + 32 * n2) + par;
        v[n2] = make_double2((double)(int64_t)src[n] * 0x1p-64,
                             (double)(int64_t)src[n + 1024] * 0x1p-64);
        if (n2) v[n2] = cmul(v[n2], c_tw32[n2]);
    }
    dft512_fwd_post(v, slots[par], lane, psi2_at<false>(psi2, 2u * lane + par),
                    psi2_at<false>(psi2, 8u * lane));
#pragma unroll
    for (int q = 0; q < 16; q++) slots[par][ffnt_pos(lane, q)] = v[q];
    __syncthreads();
    double2* dst = out + (size_t)poly * 1024;
    for (int k = threadIdx.x; k < 512; k += 64) {
        const double2 wo = cmul(slots[1][k], psi2_at<false>(psi2, 4u * k));
        dst[k] = cadd(slots[0][k], wo);
        dst[k + 512] = csub(slots[0][k], wo);
    }
}

template <bool KB, int G>
cudaError_t launch2_g(const uint32_t* lane_in, int lanes, uint64_t mu, const double2* bkf,
                      const double2* psi2, int steps, uint64_t* acc_out, uint64_t* lane_out,
                      int in_count, int mu_shift, cudaStream_t st)
{
    constexpr size_t smem = br2_smem_bytes<G>() < kSmemOneCta ? kSmemOneCta : br2_smem_bytes<G>();
    static DeviceAttrFlags attr;
    {
        const cudaError_t e = set_smem_attr_once(attr, k_br2_fp64<KB, G>, smem);
        if (e != cudaSuccess) return e;
    }
    const int blocks = (lanes + G - 1) / G;
    k_br2_fp64<KB, G><<<blocks, G * 256, smem, st>>>(lane_in, lanes, mu, bkf, psi2, steps, acc_out,
                                                     lane_out, in_count, mu_shift);
    return cudaGetLastError();
}

// ---- latency form for small batches: one lane per cluster of R CTAs on R
// SMs.  A lone lane's step is bound by one SM pulling the step's 786 KB of
// key rows (KeyBundle) from L2, and two lanes sharing an SM are held to 128
// registers per thread; here every CTA has an SM to itself, runs the lane's
// transforms on its own copy of the accumulator, multiplies only 1/R of the
// bin pairs with the key, and the inverse transforms gather the other parts
// from the peers' shared memory (distributed shared memory).  Per bin the
// arithmetic is that of k_br2_fp64, so the result is bit-identical.
constexpr int kClu2Ranks = 2;              // measured: 2 beats 4 and 8 beyond one lane
constexpr size_t kClu2Smem = kSmemOneCta;
static_assert(br2_smem_bytes<1>() <= kClu2Smem, "lvl2 cluster CTA layout");

template <bool KB, int R>
__global__ void __launch_bounds__(256, 1)
    k_br2_fp64_clu(const uint32_t* __restrict__ lane_in, int lanes, uint64_t mu,
                   const double2* __restrict__ bkf, const double2* __restrict__ psi2, int steps,
                   uint64_t* __restrict__ acc_out, uint64_t* __restrict__ lane_out, int in_count,
                   int mu_shift)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem[];
    double2* spec = reinterpret_cast<double2*>(smem);       // [8][kSlotStride]
    double2* tab = spec + 8 * kSlotStride;                  // [kPsi2Entries]
    uint64_t* acc = reinterpret_cast<uint64_t*>(tab + kPsi2Entries);  // [2][2048]
    uint16_t* abar = reinterpret_cast<uint16_t*>(acc + kTrlwe2);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int rank = (int)cluster.block_rank();
    const int l = blockIdx.x / R;
    const bool ok = l < lanes;

    for (int t = tid; t < kPsi2Entries; t += blockDim.x) tab[psi2_pos(t)] = psi2[t];
    {
        const int src = ok ? l % in_count : 0;
        const uint64_t mul = mu >> (mu_shift * (ok ? l / in_count : 0));
        const uint32_t* x = lane_in + (size_t)src * kTlwe0;
        for (int i = tid; i < kN0; i += blockDim.x)
            abar[i] = ok ? (uint16_t)((x[i] + (1u << 19)) >> 20) : 0;
        const uint32_t bar = ok ? 2u * kN2 - (x[kN0] >> 20) : 2u * kN2;
        for (int i = tid; i < kN2; i += blockDim.x) {
            acc[i] = 0;
            uint64_t v;
            if (bar == 2u * kN2)
                v = mul;
            else
                v = (((uint32_t)i < (bar & (kN2 - 1))) ^ (bar >> 11)) ? 0ull - mul : mul;
            acc[kN2 + i] = v;
        }
    }
    const double2* peer[R];
#pragma unroll
    for (int k = 0; k < R; k++) peer[k] = cluster.map_shared_rank(spec, k);
    cluster.sync();

    const int total = KB ? kN0 / 2 : kN0;
    const int nsteps = (steps < 0 || steps > total) ? total : steps;

#pragma unroll 1
    for (int p = 0; p < nsteps; p++) {
        double2 out[2][2];  // [j][bin half] of this thread's bin pair
        const double2* bk = bkf + (size_t)p * (KB ? 3 : 1) * kTrgswF2;
#pragma unroll 1
        for (int c = 0; c < 2; c++) {
            // ---- F (every rank): digits of input polynomial c, row d, parity par
            {
                const int s = warp, d = s >> 1, par = s & 1;
                const uint64_t* a = acc + c * kN2;
                const uint32_t ab = KB ? 0u : abar[p];
                const uint32_t abm = ab & (kN2 - 1), abn = ab >> 11;
                double2 v[16];
#pragma unroll
                for (int n2 = 0; n2 < 16; n2++) {
                    const int n = 2 * (lane + 32 * n2) + par;
                    uint64_t lo = a[n], hi = a[n + 1024];
                    if constexpr (!KB) {
                        uint64_t rl = a[(n - ab) & (kN2 - 1)];
                        uint64_t rh = a[(n + 1024 - ab) & (kN2 - 1)];
                        rl = (((uint32_t)n < abm) ^ abn) ? 0ull - rl : rl;
                        rh = (((uint32_t)(n + 1024) < abm) ^ abn) ? 0ull - rh : rh;
                        lo = rl - lo;
                        hi = rh - hi;
                    }
                    v[n2] = make_double2(digit2_of(lo + kDecOffset2, d),
                                         digit2_of(hi + kDecOffset2, d));
                    if (n2) v[n2] = cmul(v[n2], c_tw32[n2]);
                }
                double2* slot = spec + s * kSlotStride;
                dft512_fwd_post(v, slot, lane, psi2_at(tab, 2u * lane + par),
                                psi2_at(tab, 8u * lane));
#pragma unroll
                for (int q = 0; q < 16; q++) slot[ffnt_pos(lane, q)] = v[q];
            }
            __syncthreads();

            // ---- M (rank r): radix-2 join + key MAC of bin pairs [128 r, 128 r + 128)
            if (tid < 512 / R) {
                const int k = rank * (512 / R) + tid;  // bin pair (k, k + 512)
                const double2 w4 = psi2_at(tab, 4u * (uint32_t)k);
                double2 fac[2][3];
                if (KB) {
                    // bin k + 512: the roots of bin k times i^{2 a} (exact)
                    const uint32_t a0 = abar[2 * p];
                    const uint32_t a1 = abar[2 * p + 1];
                    const uint32_t am[3] = {a0 + a1, a0, a1};
                    const uint32_t e = 1u + 4u * (uint32_t)k;
#pragma unroll
                    for (int f = 0; f < 3; f++) {
                        fac[0][f] = psi2_at(tab, e * am[f]);
                        fac[1][f] = mul_ipow(fac[0][f], 2u * am[f]);
                    }
#pragma unroll
                    for (int h = 0; h < 2; h++)
#pragma unroll
                        for (int f = 0; f < 3; f++) fac[h][f].x -= 1.0;
                }
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int bin = k + 512 * h;
                    double2 Z[4];
#pragma unroll
                    for (int d = 0; d < 4; d++) {
                        const double2 E = spec[(2 * d) * kSlotStride + k];
                        const double2 wo = cmul(spec[(2 * d + 1) * kSlotStride + k], w4);
                        Z[d] = h ? csub(E, wo) : cadd(E, wo);
                    }
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        double2 o = c ? out[j][h] : make_double2(0.0, 0.0);
                        if (KB) {
                            double2 s0 = make_double2(0.0, 0.0), s1 = s0, s2 = s0;
#pragma unroll
                            for (int d = 0; d < 4; d++) {
                                const int r = c * 4 + d;
                                const size_t ki = ((size_t)r * 2 + j) * 1024 + bin;
                                s0 = cfma(s0, Z[d], __ldg(&bk[0 * kTrgswF2 + ki]));
                                s1 = cfma(s1, Z[d], __ldg(&bk[1 * kTrgswF2 + ki]));
                                s2 = cfma(s2, Z[d], __ldg(&bk[2 * kTrgswF2 + ki]));
                            }
                            if (j == c) {
#pragma unroll
                                for (int d = 0; d < 4; d++) {
                                    const double sc = d == 0 ? 0x1p-10 : d == 1 ? 0x1p-20
                                                    : d == 2 ? 0x1p-30 : 0x1p-40;
                                    o.x = fma(Z[d].x, sc, o.x);
                                    o.y = fma(Z[d].y, sc, o.y);
                                }
                            }
                            o = cfma(o, fac[h][0], s0);
                            o = cfma(o, fac[h][1], s1);
                            o = cfma(o, fac[h][2], s2);
                        } else {
#pragma unroll
                            for (int d = 0; d < 4; d++) {
                                const int r = c * 4 + d;
                                o = cfma(o, Z[d], __ldg(&bk[((size_t)r * 2 + j) * 1024 + bin]));
                            }
                        }
                        out[j][h] = o;
                    }
                }
                if (c == 1) {
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        spec[(2 * j) * kSlotStride + k] = cadd(out[j][0], out[j][1]);
                        spec[(2 * j + 1) * kSlotStride + k] = cmulc(csub(out[j][0], out[j][1]), w4);
                    }
                }
            }
            if (c == 0) __syncthreads();
        }
        cluster.sync();  // every rank's quarter of slots 0-3 is written

        // ---- I (every rank): gather, inverse 512-point FFT, untwist, round
        if (warp < 4) {
            const int j = (warp >> 1) & 1, par = warp & 1;
            double2 v[16];
#pragma unroll
            for (int n2 = 0; n2 < 16; n2++)
                v[n2] = peer[(n2 * 32) / (512 / R)][(2 * j + par) * kSlotStride + lane + 32 * n2];
            double2* scratch = spec + (4 + 2 * j + par) * kSlotStride;  // rows d = 2, 3 are free
            dft512_inv_raw(v, scratch, lane, psi2_at(tab, 8u * lane));
            const int k2 = lane & 15, hh = lane >> 4;
            const double2 u = psi2_at(tab, 2u * (uint32_t)(k2 + 128 * hh) + par);
            uint64_t* a = acc + j * kN2;
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int n = 2 * ffnt_pos(lane, q) + par;
                const double2 z = cmul(cmulc(v[q], u), c_utwq[q]);  // x 2^54 in c_utwq
                const uint64_t lo = to_torus64(z.x);
                const uint64_t hi = to_torus64(z.y);
                if (KB) {
                    a[n] = lo;
                    a[n + 1024] = hi;
                } else {
                    a[n] += lo;
                    a[n + 1024] += hi;
                }
            }
        }
        cluster.sync();  // the gathers are done before slots 0-3 are rewritten
    }

    if (ok && rank == 0) {
        if (acc_out)
            for (int i = tid; i < kTrlwe2; i += blockDim.x) acc_out[(size_t)l * kTrlwe2 + i] = acc[i];
        if (lane_out) {
            uint64_t* o = lane_out + (size_t)l * kTlwe2;
            for (int i = tid; i <= kN2; i += blockDim.x)
                o[i] = i == kN2 ? acc[kN2] : (i == 0 ? acc[0] : 0ull - acc[kN2 - i]);
        }
    }
}

template <bool KB, int R>
cudaError_t launch2_clu(const uint32_t* lane_in, int lanes, uint64_t mu, const double2* bkf,
                        const double2* psi2, int steps, uint64_t* acc_out, uint64_t* lane_out,
                        int in_count, int mu_shift, cudaStream_t st)
{
    static DeviceAttrFlags attr;
    {
        const cudaError_t e = set_smem_attr_once(attr, k_br2_fp64_clu<KB, R>, kClu2Smem);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(lanes * R);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = kClu2Smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = R;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_br2_fp64_clu<KB, R>, lane_in, lanes, mu, bkf, psi2, steps,
                              acc_out, lane_out, in_count, mu_shift);
}
}  // namespace

// Lanes per CTA: 1 (two CTAs per SM) unless CUFHE_BR2_LANES_PER_CTA=2 (one
// CTA per SM whose key reads serve both lanes).
cudaError_t launch_br2_fp64(bool kb, const uint32_t* lane_in, int lanes, uint64_t mu,
                            const double2* bkf, const double2* psi2, int steps, uint64_t* acc_out,
                            uint64_t* lane_out, cudaStream_t st, int in_count, int mu_shift)
{
    if (lanes <= 0) return cudaSuccess;
    if (in_count <= 0) in_count = lanes;
    {
        // batches of up to one lane per SM pair: the cluster form
        // (CUFHE_BR_CLUSTER=0 keeps one CTA per lane); a device that cannot
        // place the clusters runs the one-CTA kernel instead
        int sms = 148, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const char* ce = getenv("CUFHE_BR_CLUSTER");
        if (lanes * kClu2Ranks <= sms && !(ce && atoi(ce) == 0)) {
            const cudaError_t r =
                kb ? launch2_clu<true, kClu2Ranks>(lane_in, lanes, mu, bkf, psi2, steps, acc_out,
                                                   lane_out, in_count, mu_shift, st)
                   : launch2_clu<false, kClu2Ranks>(lane_in, lanes, mu, bkf, psi2, steps, acc_out,
                                                    lane_out, in_count, mu_shift, st);
            if (r == cudaSuccess) return r;
            cudaGetLastError();
        }
    }
    const char* e = getenv("CUFHE_BR2_LANES_PER_CTA");
    const int g = (e && atoi(e) == 2) ? 2 : 1;
    if (g == 2)
        return kb ? launch2_g<true, 2>(lane_in, lanes, mu, bkf, psi2, steps, acc_out, lane_out,
                                       in_count, mu_shift, st)
                  : launch2_g<false, 2>(lane_in, lanes, mu, bkf, psi2, steps, acc_out, lane_out,
                                        in_count, mu_shift, st);
    return kb ? launch2_g<true, 1>(lane_in, lanes, mu, bkf, psi2, steps, acc_out, lane_out,
                                   in_count, mu_shift, st)
              : launch2_g<false, 1>(lane_in, lanes, mu, bkf, psi2, steps, acc_out, lane_out,
                                    in_count, mu_shift, st);
}

cudaError_t launch_bk2_to_fft(const uint64_t* bk, int npolys, const double2* psi2, double2* out,
                              cudaStream_t st)
{
    k_bk2_to_fft<<<npolys, 64, 0, st>>>(bk, npolys, psi2, out);
    return cudaGetLastError();
}

// The FFT constants of this translation unit (fft64.cuh keeps them per file)
cudaError_t upload_fft2_constants(void)
{
    double2 w[16], t32[16], uq[16];
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < 16; k++) {
        const long double a = 2 * pi * k / 32;
        w[k] = make_double2((double)cosl(a), (double)sinl(a));
        const long double b = pi * k / 32;   // psi2^{64 k}
        t32[k] = make_double2((double)cosl(b), (double)sinl(b));
        // conj(psi2^{32 (k mod 8) + 512 (k / 8)}) 2^54: the untwist of register
        // k, the 1/1024 normalisation and the 2^64 Torus64 scale
        const long double c = -pi * ((k & 7) + 16 * (k >> 3)) / 64;
        uq[k] = make_double2((double)(cosl(c) * 0x1p54L), (double)(sinl(c) * 0x1p54L));
    }
    cudaError_t e = cudaMemcpyToSymbol(c_w32, w, sizeof(w));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tw32, t32, sizeof(t32));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_utwq, uq, sizeof(uq));
    return e;
}

}  // namespace cufhe
