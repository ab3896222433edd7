// FP64 FFNT blind rotation (the drop-in precision form) with fused
// SampleExtract.
//
// Semantics: __BlindRotate__ / __BlindRotateKeyBundle__ with Accumulate /
// AccumulateKeyBundle (include/gatebootstrapping_gpu.cuh:69-221, :801-884,
// :895-1033, :1335-1380) and __SampleExtractIndex__<P,0>
// (src/bootstrap_gpu.cu:1201-1221):
//   bar = 2N - (b >> 21)  (no rounding), abar_i = (a_i + 2^20) >> 21,
//   acc = X^bar * (0, vec(mu)),
//   non-KB step i : acc += round(IFFNT(sum_r FFNT(dec_r(X^abar acc - acc)) BK_i[r]))
//   KB pair p     : acc  = round(IFFNT(sum_r FFNT(dec_r(acc)) KB_p[r])),
//                   KB = H + bk0 (X^{a0+a1}-1) + bk1 (X^{a0}-1) + bk2 (X^{a1}-1).
//
// B200 layout.  One CTA carries G lanes (gates) through every step in
// lockstep, so each Fourier-domain key row read from L2 serves G gates
// (the reference reads the whole key per gate).  4 warps per lane:
//   phase 1  warp (g, r): digits of row r of lane g, fold + twist, forward
//            512-point FFT (one warp per transform, fft64.cuh) -> spec[g][r]
//   phase 2  thread f (frequency bin): key multiply-accumulate for all G lanes;
//            key words are read once per CTA with 128-bit loads; the KeyBundle
//            factors X^a - 1 are evaluated from a 2N-entry root table
//            (psi^{(1+4f) a} - 1) instead of the reference's 16 MB xai table
//   phase 3  warp (g, j): inverse FFT, untwist, round, write acc[g][j]
// Epilogue: SampleExtract straight from shared memory to the lane output.
// Batches of up to 16 lanes run the latency form k_br_fp64_clu instead: one
// lane per cluster of four CTAs on four SMs, each multiplying a quarter of the
// bins with the key (a lone lane is bound by one SM's L2 bandwidth for the
// 196 KB of key rows per step) and gathering the other quarters through
// distributed shared memory for the inverse transforms.
#include <stdlib.h>

#include <cooperative_groups.h>

#include "engine.h"
#include "fft64.cuh"

namespace cufhe {

namespace {

constexpr int kDefaultBrGates = 2;
constexpr int kAbarStride = 640;
constexpr uint32_t kDecOffset = (128u << 24) + (128u << 16) + (1u << 15);  // offsetgen + round

template <int G>
constexpr size_t br_smem_bytes()
{
    return sizeof(double2) * G * 4 * kSlotStride + sizeof(double2) * kN +
           sizeof(uint32_t) * G * kTrlwe + sizeof(uint16_t) * G * kAbarStride;
}

// Word of coefficient n (0 <= n < 2N) of a lane's accumulator in shared
// memory.  The KeyBundle form flips bit 4 when bit 7 is set: the inverse
// transforms store coefficients n and n + 128 from lanes l and l + 16 in one
// instruction, which would otherwise fall in the same bank; the forward
// transforms' reads of 32 consecutive coefficients stay conflict-free.  (The
// plain form keeps the natural order: its rotated reads X^a acc start
// anywhere.)
template <bool KB>
__device__ __forceinline__ int acc_ix(int n)
{
    return KB ? n ^ (((n >> 7) & 1) << 4) : n;
}

// signed digit d (0 = most significant) of an offset Torus32 value
__device__ __forceinline__ double digit_of(uint32_t t, int d)
{
    return (double)((int32_t)((t >> (24 - 8 * d)) & 255u) - 128);
}

template <bool KB, int G>
__global__ void __launch_bounds__(G * 128, G == 1 ? 3 : (G == 2 ? 2 : 1)) k_br_fp64(const uint32_t* __restrict__ lane_in, int lanes,
                                                     uint32_t mu, const double2* __restrict__ bkf,
                                                     const double2* __restrict__ psi,
                                                     const double2* __restrict__ tw512, int steps,
                                                     uint32_t* __restrict__ acc_out,
                                                     uint32_t* __restrict__ lane_out)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double2* spec = reinterpret_cast<double2*>(smem);
    double2* psi_s = spec + G * 4 * kSlotStride;  // root table, interleaved (psi_pos)
    uint32_t* acc = reinterpret_cast<uint32_t*>(psi_s + kN);
    uint16_t* abar = reinterpret_cast<uint16_t*>(acc + G * kTrlwe);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int lane_base = blockIdx.x * G;

    for (int t = tid; t < kN; t += blockDim.x) psi_s[psi_pos((uint32_t)t)] = psi[t];
    // ---- prologue: modulus switch and test vector (RotatedTestVector)
#pragma unroll 1
    for (int g = 0; g < G; g++) {
        const int l = lane_base + g;
        const bool ok = l < lanes;
        const uint32_t* x = lane_in + (size_t)(ok ? l : 0) * kTlwe0;
        for (int i = tid; i < kN0; i += blockDim.x)
            abar[g * kAbarStride + i] = ok ? (uint16_t)((x[i] + (1u << 20)) >> 21) : 0;
        const uint32_t bar = ok ? 2u * kN - (x[kN0] >> 21) : 2u * kN;
        for (int i = tid; i < kN; i += blockDim.x) {
            acc[g * kTrlwe + acc_ix<KB>(i)] = 0;
            uint32_t v;
            if (bar == 2u * kN)
                v = mu;
            else
                v = (((uint32_t)i < (bar & (kN - 1))) ^ (bar >> 10)) ? 0u - mu : mu;
            acc[g * kTrlwe + acc_ix<KB>(kN + i)] = v;
        }
    }
    __syncthreads();

    const int total = KB ? kN0 / 2 : kN0;
    const int nsteps = (steps < 0 || steps > total) ? total : steps;
    constexpr size_t kTrgswF = 4 * 2 * kHalfN;  // double2 per Fourier TRGSW

#pragma unroll 1
    for (int p = 0; p < nsteps; p++) {
        // ---- phase 1: decompose + fold + twist + forward FFT, warp (g, r)
        {
            const int g = warp >> 2, r = warp & 3, j = r >> 1, d = r & 1;
            const uint32_t* a = acc + g * kTrlwe + j * kN;
            double2 v[16];
            const uint32_t ab = KB ? 0u : abar[g * kAbarStride + p];
            const uint32_t abm = ab & (kN - 1), abn = ab >> 10;
#pragma unroll
            for (int n2 = 0; n2 < 16; n2++) {
                const int n = lane + 32 * n2;
                uint32_t lo = a[acc_ix<KB>(n)], hi = a[acc_ix<KB>(n + kHalfN)];
                if (!KB) {
                    // X^abar acc - acc (include/gatebootstrapping_gpu.cuh:114-138)
                    uint32_t rl = a[(n - ab) & (kN - 1)];
                    uint32_t rh = a[(n + kHalfN - ab) & (kN - 1)];
                    rl = (((uint32_t)n < abm) ^ abn) ? 0u - rl : rl;
                    rh = (((uint32_t)(n + kHalfN) < abm) ^ abn) ? 0u - rh : rh;
                    lo = rl - lo;
                    hi = rh - hi;
                }
                v[n2] = make_double2(digit_of(lo + kDecOffset, d), digit_of(hi + kDecOffset, d));
            }
            double2* slot = spec + (g * 4 + r) * kSlotStride;
            ffnt_forward_warp(v, slot, psi_s, lane);
#pragma unroll
            for (int q = 0; q < 16; q++) slot[ffnt_pos(lane, q)] = v[q];
        }
        __syncthreads();

        // ---- phase 2: key multiply-accumulate, thread f = frequency bin.
        // One (bin, output polynomial) item at a time with all twelve key
        // words of the item (rows x keys) loaded before any is used: the
        // phase is bound by the latency of the key rows from L2, and this
        // keeps 12 loads per thread in flight (a rows-outermost loop with both
        // outputs' accumulators live leaves room for only one row's 6).  The
        // output of polynomial 0 overwrites row 0's spectrum, which polynomial
        // 1 still reads, so it is held in registers until both are done.  Per
        // bin and output the additions run in the same order as in
        // k_br_fp64_clu (rows 0..3, then H, x01, x0, x1): bit-identical.
        if (KB) {
            const double2* bk = bkf + (size_t)p * 3 * kTrgswF;
            // KeyBundle roots psi^{(1 + 4 f) a} (a = a0 + a1, a0, a1) of the
            // thread's first bin.  With two lanes per CTA the thread's bins
            // are f and f + 256, and psi^{(1 + 4 (f + 256)) a} = (-1)^a
            // psi^{(1 + 4 f) a} exactly (a sign flip), so the roots are
            // gathered once per step; the table gathers are bank-conflicted
            // for even a.  Other lane counts gather per bin.
            double2 root[G][3];
            uint32_t odd[G];
            if (G == 2) {
                const uint32_t ef = 1u + 4u * (uint32_t)tid;
#pragma unroll
                for (int g = 0; g < G; g++) {
                    const uint32_t a0 = abar[g * kAbarStride + 2 * p];
                    const uint32_t a1 = abar[g * kAbarStride + 2 * p + 1];
                    root[g][0] = psi_at(psi_s, ef * (a0 + a1));
                    root[g][1] = psi_at(psi_s, ef * a0);
                    root[g][2] = psi_at(psi_s, ef * a1);
                    odd[g] = (((a0 + a1) & 1u) << 0) | ((a0 & 1u) << 1) | ((a1 & 1u) << 2);
                }
            }
#pragma unroll 1
            for (int f = tid; f < kHalfN; f += blockDim.x) {
                const uint32_t ef = 1u + 4u * (uint32_t)f;
                double2 o0[G];
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    double2 b[4][3];
#pragma unroll
                    for (int r = 0; r < 4; r++)
#pragma unroll
                        for (int e = 0; e < 3; e++)
                            b[r][e] = __ldg(&bk[((e * 4 + r) * 2 + j) * kHalfN + f]);
#pragma unroll
                    for (int g = 0; g < G; g++) {
                        double2 D[4], sum[3];
#pragma unroll
                        for (int r = 0; r < 4; r++) D[r] = spec[(g * 4 + r) * kSlotStride + f];
#pragma unroll
                        for (int r = 0; r < 4; r++)
#pragma unroll
                            for (int e = 0; e < 3; e++)
                                sum[e] = r == 0 ? cfma(make_double2(0.0, 0.0), D[r], b[r][e])
                                                : cfma(sum[e], D[r], b[r][e]);
                        // FFNT(H 2^-32) = 2^-8 (d = 0), 2^-16 (d = 1) on poly j
                        double2 o = make_double2(fma(D[2 * j].x, 0x1p-8, D[2 * j + 1].x * 0x1p-16),
                                                 fma(D[2 * j].y, 0x1p-8, D[2 * j + 1].y * 0x1p-16));
                        double2 x01, x0, x1;
                        if (G == 2) {
                            x01 = root[g][0];
                            x0 = root[g][1];
                            x1 = root[g][2];
                        } else {
                            const uint32_t a0 = abar[g * kAbarStride + 2 * p];
                            const uint32_t a1 = abar[g * kAbarStride + 2 * p + 1];
                            x01 = psi_at(psi_s, ef * (a0 + a1));
                            x0 = psi_at(psi_s, ef * a0);
                            x1 = psi_at(psi_s, ef * a1);
                        }
                        x0.x -= 1.0;
                        x1.x -= 1.0;
                        x01.x -= 1.0;
                        o = cfma(o, x01, sum[0]);
                        o = cfma(o, x0, sum[1]);
                        o = cfma(o, x1, sum[2]);
                        if (j == 0) {
                            o0[g] = o;
                        } else {
                            spec[(g * 4 + 0) * kSlotStride + f] = o0[g];
                            spec[(g * 4 + 1) * kSlotStride + f] = o;
                        }
                    }
                }
                if (G == 2) {
#pragma unroll
                    for (int g = 0; g < G; g++)
#pragma unroll
                        for (int e = 0; e < 3; e++)
                            if ((odd[g] >> e) & 1u) {
                                root[g][e].x = -root[g][e].x;
                                root[g][e].y = -root[g][e].y;
                            }
                }
            }
        } else {
            const double2* bk = bkf + (size_t)p * kTrgswF;
            for (int f = tid; f < kHalfN; f += blockDim.x) {
                double2 o[G][2];
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    double2 b[2];
#pragma unroll
                    for (int j = 0; j < 2; j++) b[j] = __ldg(&bk[(r * 2 + j) * kHalfN + f]);
#pragma unroll
                    for (int g = 0; g < G; g++) {
                        const double2 D = spec[(g * 4 + r) * kSlotStride + f];
#pragma unroll
                        for (int j = 0; j < 2; j++)
                            o[g][j] = r == 0 ? cfma(make_double2(0.0, 0.0), D, b[j])
                                             : cfma(o[g][j], D, b[j]);
                    }
                }
#pragma unroll
                for (int g = 0; g < G; g++) {
                    spec[(g * 4 + 0) * kSlotStride + f] = o[g][0];
                    spec[(g * 4 + 1) * kSlotStride + f] = o[g][1];
                }
            }
        }
        __syncthreads();

        // ---- phase 3: inverse FFT + untwist + round, warp (g, j)
        if (warp < 2 * G) {
            const int g = warp >> 1, j = warp & 1;
            double2* slot = spec + (g * 4 + j) * kSlotStride;
            double2 v[16];
#pragma unroll
            for (int n2 = 0; n2 < 16; n2++) v[n2] = slot[lane + 32 * n2];
            __syncwarp();
            ffnt_inverse_warp(v, slot, psi_s, lane);
            uint32_t* a = acc + g * kTrlwe + j * kN;
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int n = ffnt_pos(lane, q);
                // already untwisted and scaled to Torus32 units (x 2^23)
                const double2 u = v[q];
                const uint32_t lo = (uint32_t)__double2ll_rn(u.x);
                const uint32_t hi = (uint32_t)__double2ll_rn(u.y);
                if (KB) {
                    a[acc_ix<KB>(n)] = lo;
                    a[acc_ix<KB>(n + kHalfN)] = hi;
                } else {
                    a[n] += lo;
                    a[n + kHalfN] += hi;
                }
            }
        }
        __syncthreads();
    }

    // ---- epilogue: accumulator and/or SampleExtract (index 0)
    for (int g = 0; g < G; g++) {
        const int l = lane_base + g;
        if (l >= lanes) break;
        const uint32_t* a = acc + g * kTrlwe;
        if (acc_out)
            for (int i = tid; i < kTrlwe; i += blockDim.x)
                acc_out[(size_t)l * kTrlwe + i] = a[acc_ix<KB>(i)];
        if (lane_out) {
            uint32_t* o = lane_out + (size_t)l * kTlwe1;
            for (int i = tid; i <= kN; i += blockDim.x)
                o[i] = i == kN ? a[acc_ix<KB>(kN)] : (i == 0 ? a[0] : 0u - a[acc_ix<KB>(kN - i)]);
        }
    }
}

// BK polynomial -> Fourier domain: read as signed int32, scale 2^-32, fold,
// twist, forward FFT (src/bootstrap_gpu.cu:59-112).  One warp per polynomial.
__global__ void __launch_bounds__(128) k_bk_to_fft(const uint32_t* __restrict__ bk, int npolys,
                                                   const double2* __restrict__ psi,
                                                   const double2* __restrict__ tw512,
                                                   double2* __restrict__ out)
{
    __shared__ __align__(16) double2 tiles[4][kSlotStride];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int poly = blockIdx.x * 4 + warp;
    if (poly >= npolys) return;
    const uint32_t* src = bk + (size_t)poly * kN;
    double2 v[16];
#pragma unroll
    for (int n2 = 0; n2 < 16; n2++) {
        const int n = lane + 32 * n2;
        const double2 z = make_double2((double)(int32_t)src[n] * 0x1p-32,
                                       (double)(int32_t)src[n + kHalfN] * 0x1p-32);
        v[n2] = cmul(z, __ldg(&psi[n]));
    }
    fft512_warp<1>(v, tiles[warp], tw512, lane);
    double2* dst = out + (size_t)poly * kHalfN;
#pragma unroll
    for (int m = 0; m < 16; m++) dst[(lane & 15) + 16 * m + 256 * (lane >> 4)] = v[m];
}

template <bool KB, int G>
cudaError_t launch_g(const uint32_t* lane_in, int lanes, uint32_t mu, const double2* bkf,
                     const Fp64Tables& t, int steps, uint32_t* acc_out, uint32_t* lane_out,
                     cudaStream_t st)
{
    constexpr size_t smem = br_smem_bytes<G>();
    static DeviceAttrFlags attr;
    {
        const cudaError_t e = set_smem_attr_once(attr, k_br_fp64<KB, G>, smem);
        if (e != cudaSuccess) return e;
    }
    const int blocks = (lanes + G - 1) / G;
    k_br_fp64<KB, G><<<blocks, G * 128, smem, st>>>(lane_in, lanes, mu, bkf, t.psi, t.tw512, steps,
                                                    acc_out, lane_out);
    return cudaGetLastError();
}

// ---- latency form for small batches: one lane per cluster of four CTAs on
// four SMs.  A single lane's step is bound by the rate at which one SM pulls
// the step's key rows from L2 (196 KB per KeyBundle step); here every CTA of
// the cluster runs the lane's transforms (redundantly, on its own copy of the
// accumulator) but multiplies only its quarter of the frequency bins with the
// key, and the inverse transforms gather the four quarters from the peers'
// shared memory (distributed shared memory).  The arithmetic of every bin is
// that of k_br_fp64, so the result is bit-identical.
constexpr int kCluRanks = 4;
constexpr int kCluMaxLanes = 16;         // measured: faster than one CTA per lane up to 16 lanes
constexpr size_t kCluSmem = 120 * 1024;  // > half an SM: one CTA per SM

template <bool KB>
__global__ void __cluster_dims__(kCluRanks, 1, 1) __launch_bounds__(128, 1)
    k_br_fp64_clu(const uint32_t* __restrict__ lane_in, int lanes, uint32_t mu,
                  const double2* __restrict__ bkf, const double2* __restrict__ psi, int steps,
                  uint32_t* __restrict__ acc_out, uint32_t* __restrict__ lane_out)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem[];
    double2* spec = reinterpret_cast<double2*>(smem);
    double2* psi_s = spec + 4 * kSlotStride;
    uint32_t* acc = reinterpret_cast<uint32_t*>(psi_s + kN);
    uint16_t* abar = reinterpret_cast<uint16_t*>(acc + kTrlwe);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int rank = (int)cluster.block_rank();
    const int l = blockIdx.x / kCluRanks;
    const bool ok = l < lanes;

    for (int t = tid; t < kN; t += blockDim.x) psi_s[psi_pos((uint32_t)t)] = psi[t];
    {
        const uint32_t* x = lane_in + (size_t)(ok ? l : 0) * kTlwe0;
        for (int i = tid; i < kN0; i += blockDim.x)
            abar[i] = ok ? (uint16_t)((x[i] + (1u << 20)) >> 21) : 0;
        const uint32_t bar = ok ? 2u * kN - (x[kN0] >> 21) : 2u * kN;
        for (int i = tid; i < kN; i += blockDim.x) {
            acc[i] = 0;
            uint32_t v;
            if (bar == 2u * kN)
                v = mu;
            else
                v = (((uint32_t)i < (bar & (kN - 1))) ^ (bar >> 10)) ? 0u - mu : mu;
            acc[kN + i] = v;
        }
    }
    // the peers' transform slots 0 and 1 (the multiply-accumulate results)
    const double2* peer[kCluRanks];
#pragma unroll
    for (int k = 0; k < kCluRanks; k++) peer[k] = cluster.map_shared_rank(spec, k);
    cluster.sync();

    const int total = KB ? kN0 / 2 : kN0;
    const int nsteps = (steps < 0 || steps > total) ? total : steps;
    constexpr size_t kTrgswF = 4 * 2 * kHalfN;

#pragma unroll 1
    for (int p = 0; p < nsteps; p++) {
        // ---- phase 1 (every rank): decompose + fold + twist + forward FFT, warp r
        {
            const int r = warp, j = r >> 1, d = r & 1;
            const uint32_t* a = acc + j * kN;
            double2 v[16];
            const uint32_t ab = KB ? 0u : abar[p];
            const uint32_t abm = ab & (kN - 1), abn = ab >> 10;
#pragma unroll
            for (int n2 = 0; n2 < 16; n2++) {
                const int n = lane + 32 * n2;
                uint32_t lo = a[n], hi = a[n + kHalfN];
                if (!KB) {
                    uint32_t rl = a[(n - ab) & (kN - 1)];
                    uint32_t rh = a[(n + kHalfN - ab) & (kN - 1)];
                    rl = (((uint32_t)n < abm) ^ abn) ? 0u - rl : rl;
                    rh = (((uint32_t)(n + kHalfN) < abm) ^ abn) ? 0u - rh : rh;
                    lo = rl - lo;
                    hi = rh - hi;
                }
                v[n2] = make_double2(digit_of(lo + kDecOffset, d), digit_of(hi + kDecOffset, d));
            }
            double2* slot = spec + r * kSlotStride;
            ffnt_forward_warp(v, slot, psi_s, lane);
#pragma unroll
            for (int q = 0; q < 16; q++) slot[ffnt_pos(lane, q)] = v[q];
        }
        __syncthreads();

        // ---- phase 2 (rank k): key multiply-accumulate of bins [128 k, 128 k + 128)
        {
            const int f = rank * 128 + tid;
            double2 D[4];
#pragma unroll
            for (int r = 0; r < 4; r++) D[r] = spec[r * kSlotStride + f];
            double2 out0;
            if (KB) {
                const double2* bk = bkf + (size_t)p * 3 * kTrgswF;
                const uint32_t ef = 1u + 4u * (uint32_t)f;
                const uint32_t a0 = abar[2 * p], a1 = abar[2 * p + 1];
                double2 x0 = psi_at(psi_s, ef * a0);
                double2 x1 = psi_at(psi_s, ef * a1);
                double2 x01 = psi_at(psi_s, ef * (a0 + a1));
                x0.x -= 1.0;
                x1.x -= 1.0;
                x01.x -= 1.0;
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    double2 b[3][4];
#pragma unroll
                    for (int e = 0; e < 3; e++)
#pragma unroll
                        for (int r = 0; r < 4; r++)
                            b[e][r] = __ldg(&bk[((e * 4 + r) * 2 + j) * kHalfN + f]);
                    double2 s0 = make_double2(0.0, 0.0), s1 = s0, s2 = s0;
#pragma unroll
                    for (int r = 0; r < 4; r++) {
                        s0 = cfma(s0, D[r], b[0][r]);
                        s1 = cfma(s1, D[r], b[1][r]);
                        s2 = cfma(s2, D[r], b[2][r]);
                    }
                    double2 o = make_double2(fma(D[2 * j].x, 0x1p-8, D[2 * j + 1].x * 0x1p-16),
                                             fma(D[2 * j].y, 0x1p-8, D[2 * j + 1].y * 0x1p-16));
                    o = cfma(o, x01, s0);
                    o = cfma(o, x0, s1);
                    o = cfma(o, x1, s2);
                    if (j == 0)
                        out0 = o;
                    else {
                        spec[0 * kSlotStride + f] = out0;
                        spec[1 * kSlotStride + f] = o;
                    }
                }
            } else {
                const double2* bk = bkf + (size_t)p * kTrgswF;
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    double2 o = make_double2(0.0, 0.0);
#pragma unroll
                    for (int r = 0; r < 4; r++)
                        o = cfma(o, D[r], __ldg(&bk[(r * 2 + j) * kHalfN + f]));
                    if (j == 0)
                        out0 = o;
                    else {
                        spec[0 * kSlotStride + f] = out0;
                        spec[1 * kSlotStride + f] = o;
                    }
                }
            }
        }
        cluster.sync();  // every rank's quarter of slots 0 and 1 is written

        // ---- phase 3 (every rank): gather, inverse FFT, untwist, round, warp j
        if (warp < 2) {
            const int j = warp;
            double2 v[16];
#pragma unroll
            for (int n2 = 0; n2 < 16; n2++)
                v[n2] = peer[n2 >> 2][j * kSlotStride + lane + 32 * n2];
            double2* scratch = spec + (2 + j) * kSlotStride;  // rows 2, 3 are free now
            ffnt_inverse_warp(v, scratch, psi_s, lane);
            uint32_t* a = acc + j * kN;
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int n = ffnt_pos(lane, q);
                const double2 u = v[q];  // untwisted, in Torus32 units
                const uint32_t lo = (uint32_t)__double2ll_rn(u.x);
                const uint32_t hi = (uint32_t)__double2ll_rn(u.y);
                if (KB) {
                    a[n] = lo;
                    a[n + kHalfN] = hi;
                } else {
                    a[n] += lo;
                    a[n + kHalfN] += hi;
                }
            }
        }
        cluster.sync();  // the gathers are done before slots 0 and 1 are rewritten
    }

    if (ok && rank == 0) {
        if (acc_out)
            for (int i = tid; i < kTrlwe; i += blockDim.x) acc_out[(size_t)l * kTrlwe + i] = acc[i];
        if (lane_out) {
            uint32_t* o = lane_out + (size_t)l * kTlwe1;
            for (int i = tid; i <= kN; i += blockDim.x)
                o[i] = i == kN ? acc[kN] : (i == 0 ? acc[0] : 0u - acc[kN - i]);
        }
    }
}

template <bool KB>
cudaError_t launch_clu(const uint32_t* lane_in, int lanes, uint32_t mu, const double2* bkf,
                       const Fp64Tables& t, int steps, uint32_t* acc_out, uint32_t* lane_out,
                       cudaStream_t st)
{
    static DeviceAttrFlags attr;
    {
        const cudaError_t e = set_smem_attr_once(attr, k_br_fp64_clu<KB>, kCluSmem);
        if (e != cudaSuccess) return e;
    }
    k_br_fp64_clu<KB><<<lanes * kCluRanks, 128, kCluSmem, st>>>(lane_in, lanes, mu, bkf, t.psi, steps,
                                                              acc_out, lane_out);
    return cudaGetLastError();
}
}  // namespace

// Lanes per CTA: 1 (three CTAs per SM), 2 (two CTAs per SM, whose phases
// overlap) or 4 (one CTA per SM, key rows shared by 4 lanes).  CUFHE_BR_LANES_PER_CTA overrides the
// default for tuning.
static int br_lanes_per_cta()
{
    static int g = 0;
    if (!g) {
        const char* e = getenv("CUFHE_BR_LANES_PER_CTA");
        g = (e && atoi(e) == 4) ? 4 : (e && atoi(e) == 2) ? 2 : (e && atoi(e) == 1) ? 1 : kDefaultBrGates;
    }
    return g;
}

namespace {
struct BrTuning {
    int n = 0;
    int bound[32];
    int g[32];
};
BrTuning g_br_tuning[64];
}  // namespace

void br_fp64_set_tuning(int dev, int n, const int* bound, const int* g)
{
    BrTuning& t = g_br_tuning[dev & 63];
    t.n = n < 0 ? 0 : (n > 32 ? 32 : n);
    for (int i = 0; i < t.n; i++) {
        t.bound[i] = bound[i];
        t.g[i] = g[i];
    }
}

int br_fp64_get_tuning(int dev, int* bound, int* g, int cap)
{
    const BrTuning& t = g_br_tuning[dev & 63];
    for (int i = 0; i < t.n && i < cap; i++) {
        bound[i] = t.bound[i];
        g[i] = t.g[i];
    }
    return t.n;
}

cudaError_t launch_br_fp64(bool kb, const uint32_t* lane_in, int lanes, uint32_t mu,
                           const double2* bkf, const Fp64Tables& t, int steps, uint32_t* acc_out,
                           uint32_t* lane_out, cudaStream_t st)
{
    if (lanes <= 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    int g;
    const BrTuning& tun = g_br_tuning[dev & 63];
    if (getenv("CUFHE_BR_LANES_PER_CTA")) {
        g = br_lanes_per_cta();
    } else if (tun.n > 0) {
        int i = 0;
        while (i + 1 < tun.n && lanes > tun.bound[i]) i++;
        g = tun.g[i];
    } else {
        // untuned: one lane per CTA (3 CTAs per SM) while the batch fits one
        // wave, which minimises latency; larger ones: two lanes per CTA
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g = lanes <= 3 * sms ? 1 : kDefaultBrGates;
    }
    return launch_br_fp64_g(g, kb, lane_in, lanes, mu, bkf, t, steps, acc_out, lane_out, st);
}

cudaError_t launch_br_fp64_g(int g, bool kb, const uint32_t* lane_in, int lanes, uint32_t mu,
                             const double2* bkf, const Fp64Tables& t, int steps,
                             uint32_t* acc_out, uint32_t* lane_out, cudaStream_t st)
{
    if (lanes <= 0) return cudaSuccess;
    if (g == 1 && lanes <= kCluMaxLanes) {
        // small batches: one lane per cluster of four SMs (CUFHE_BR_CLUSTER=0
        // keeps one CTA per lane); a device that cannot place the clusters
        // runs the one-CTA kernel instead
        int sms = 148, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const char* e = getenv("CUFHE_BR_CLUSTER");
        if (lanes * kCluRanks <= sms && !(e && atoi(e) == 0)) {
            const cudaError_t r =
                kb ? launch_clu<true>(lane_in, lanes, mu, bkf, t, steps, acc_out, lane_out, st)
                   : launch_clu<false>(lane_in, lanes, mu, bkf, t, steps, acc_out, lane_out, st);
            if (r == cudaSuccess) return r;
            cudaGetLastError();
        }
    }
    if (g == 1)
        return kb ? launch_g<true, 1>(lane_in, lanes, mu, bkf, t, steps, acc_out, lane_out, st)
                  : launch_g<false, 1>(lane_in, lanes, mu, bkf, t, steps, acc_out, lane_out, st);
    if (g == 2)
        return kb ? launch_g<true, 2>(lane_in, lanes, mu, bkf, t, steps, acc_out, lane_out, st)
                  : launch_g<false, 2>(lane_in, lanes, mu, bkf, t, steps, acc_out, lane_out, st);
    return kb ? launch_g<true, 4>(lane_in, lanes, mu, bkf, t, steps, acc_out, lane_out, st)
              : launch_g<false, 4>(lane_in, lanes, mu, bkf, t, steps, acc_out, lane_out, st);
}

cudaError_t launch_bk_to_fft(const uint32_t* bk, int npolys, const Fp64Tables& t, double2* out,
                             cudaStream_t st)
{
    k_bk_to_fft<<<(npolys + 3) / 4, 128, 0, st>>>(bk, npolys, t.psi, t.tw512, out);
    return cudaGetLastError();
}

cudaError_t upload_fft_constants(void)
{
    double2 w[16], t32[16], uq[16];
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < 16; k++) {
        const long double a = 2 * pi * k / 32;
        w[k] = make_double2((double)cosl(a), (double)sinl(a));
        const long double b = pi * k / 32;  // psi^{32 k}
        t32[k] = make_double2((double)cosl(b), (double)sinl(b));
        // conj(psi^{16 (k mod 8) + 256 (k / 8)}) 2^23
        const long double c = -pi * (16 * (k & 7) + 256 * (k >> 3)) / 1024;
        uq[k] = make_double2((double)(cosl(c) * 0x1p23L), (double)(sinl(c) * 0x1p23L));
    }
    cudaError_t e = cudaMemcpyToSymbol(c_w32, w, sizeof(w));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tw32, t32, sizeof(t32));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_utwq, uq, sizeof(uq));
    return e;
}

}  // namespace cufhe
