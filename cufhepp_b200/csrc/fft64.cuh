// FP64 negacyclic FFNT for N = 1024 (512-point complex transform), one warp
// per polynomial.
//
// Same transform as the reference's GPU-FFT backend (fold, twist, N/2-point
// FFT with roots e^{+2 pi i k/(N/2)}, inverse with conjugate roots, untwist
// with 1/(N/2) folded in: src/ntt_small_modulus.cu:207-244,
// include/ntt_small_modulus.cuh:977-1182), restructured for a warp:
//
//   512 = 16 x 32.  Lane n1 holds x[n1 + 32 n2], n2 = 0..15, in registers.
//   1. 16-point DFT over n2 in registers (radix 4 x 4).
//   2. twiddle w512^(n1 k2) (table, coalesced per lane).
//   3. transpose through a padded 16 x 33 shared-memory tile (conflict-free).
//   4. lane (k2 + 16 h) holds the n1 = h + 2m half of sequence k2; 16-point
//      DFT over m in registers.
//   5. one radix-2 stage across lanes l and l ^ 16 (warp shuffle).
//   Output: lane (k2 + 16 h), register m holds bin k2 + 16 m + 256 h
//   (fft512_warp: key conversion, CMUX).  The blind-rotation transforms
//   (ffnt_forward_warp / ffnt_inverse_warp and the N = 2048 halves) run step
//   5 with both lanes of a pair busy (radix2_pair) and leave register q at
//   ffnt_pos(lane, q) instead.
//
// The reference runs one 512-point FFT per CTA with 256 threads and
// __syncthreads between stages; here a warp owns a whole transform and only
// synchronises with __syncwarp, so 16+ transforms proceed independently per
// SM.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cufhe {

constexpr int kHalfN = 512;
constexpr int kSlotStride = 528;  // double2 per transform slot (16 x 33 tile)

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ double2 cfma(double2 acc, double2 a, double2 b)
{
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
// multiply by S*i, S = +1 (forward) or -1 (inverse)
template <int S>
__device__ __forceinline__ double2 mul_si(double2 a)
{
    return S > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// Radix-2 butterfly across lanes l and l ^ 16 (h = l >> 4): lanes h = 0 hold
// E0, lanes h = 1 hold E1; afterwards h = 0 holds E0 + w E1 and h = 1 holds
// E0 - w E1.  Lanes h = 1 multiply by w, and every lane finishes with
// o + sg * t as one FMA per component (sg = +-1) instead of computing both
// the sum and the difference and selecting one; an FMA by +-1 rounds like
// the add or subtract it replaces, so the results are the same bit for bit.
__device__ __forceinline__ double2 radix2_xlane(double2 v, double2 w, int h)
{
    const double sg = h ? -1.0 : 1.0;
    const double2 t = h ? cmul(v, w) : v;
    double2 o;
    o.x = __shfl_xor_sync(0xffffffffu, t.x, 16);
    o.y = __shfl_xor_sync(0xffffffffu, t.y, 16);
    return make_double2(fma(sg, t.x, o.x), fma(sg, t.y, o.y));
}

// In-place 4-point DFT with root S*i.
template <int S>
__device__ __forceinline__ void dft4(double2& u0, double2& u1, double2& u2, double2& u3)
{
    const double2 t0 = cadd(u0, u2), t1 = csub(u0, u2);
    const double2 t2 = cadd(u1, u3), t3 = mul_si<S>(csub(u1, u3));
    u0 = cadd(t0, t2);
    u2 = csub(t0, t2);
    u1 = cadd(t1, t3);
    u3 = csub(t1, t3);
}

// In-place 16-point DFT, natural order in and out:
//   X[k] = sum_n x[n] e^{S 2 pi i n k / 16}
// radix 4 x 4: n = 4a + b, k = c + 4d.
template <int S>
__device__ __forceinline__ void dft16(double2 (&v)[16])
{
    constexpr double C1 = 0.92387953251128675613; // cos(pi/8)
    constexpr double S1 = 0.38268343236508977173; // sin(pi/8)
    constexpr double R2 = 0.70710678118654752440; // cos(pi/4)
#pragma unroll
    for (int b = 0; b < 4; b++) dft4<S>(v[b], v[4 + b], v[8 + b], v[12 + b]);
    // now v[4c + b] = y[b][c]; twiddle by w^(b c), w = e^{S 2 pi i/16}
    // (b, c) = (1,1): w, (1,2): w^2, (1,3): w^3, (2,1): w^2, (2,2): w^4 = S i,
    // (2,3): w^6, (3,1): w^3, (3,2): w^6, (3,3): w^9
    const double2 w1 = make_double2(C1, S * S1);
    const double2 w3 = make_double2(S1, S * C1);
    const double2 w9 = make_double2(-C1, -S * S1);
    auto mw2 = [](double2 a) {  // * (R2, S R2)
        return make_double2(R2 * (a.x - S * a.y), R2 * (a.y + S * a.x));
    };
    auto mw6 = [](double2 a) {  // * (-R2, S R2)
        return make_double2(-R2 * (a.x + S * a.y), R2 * (S * a.x - a.y));
    };
    v[4 * 1 + 1] = cmul(v[4 * 1 + 1], w1);
    v[4 * 2 + 1] = mw2(v[4 * 2 + 1]);
    v[4 * 3 + 1] = cmul(v[4 * 3 + 1], w3);
    v[4 * 1 + 2] = mw2(v[4 * 1 + 2]);
    v[4 * 2 + 2] = mul_si<S>(v[4 * 2 + 2]);
    v[4 * 3 + 2] = mw6(v[4 * 3 + 2]);
    v[4 * 1 + 3] = cmul(v[4 * 1 + 3], w3);
    v[4 * 2 + 3] = mw6(v[4 * 2 + 3]);
    v[4 * 3 + 3] = cmul(v[4 * 3 + 3], w9);
    // 4-point DFT over b for each c: X[c + 4d]
    double2 o[16];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        double2 u0 = v[4 * c + 0], u1 = v[4 * c + 1], u2 = v[4 * c + 2], u3 = v[4 * c + 3];
        dft4<S>(u0, u1, u2, u3);
        o[c + 0] = u0;
        o[c + 4] = u1;
        o[c + 8] = u2;
        o[c + 12] = u3;
    }
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = o[k];
}

// Twiddles of the 32-point stage: e^{2 pi i k / 32}, k = 0..15
static __constant__ double2 c_w32[16];

// Warp-level 512-point DFT with root e^{S 2 pi i / 512}.
//   in : v[n2] = x[lane + 32 n2]
//   out: v[m]  = X[(lane & 15) + 16 m + 256 (lane >> 4)]
// tile: this warp's shared slot (>= 528 double2), free on entry; tw512:
// global table tw512[k2 * 32 + n1] = e^{2 pi i n1 k2 / 512}.
template <int S>
__device__ __forceinline__ void fft512_warp(double2 (&v)[16], double2* tile,
                                            const double2* __restrict__ tw512, int lane)
{
    dft16<S>(v);
#pragma unroll
    for (int k2 = 1; k2 < 16; k2++) {
        const double2 w = __ldg(&tw512[k2 * 32 + lane]);
        v[k2] = S > 0 ? cmul(v[k2], w) : cmulc(v[k2], w);
    }
#pragma unroll
    for (int k2 = 0; k2 < 16; k2++) tile[k2 * 33 + lane] = v[k2];
    __syncwarp();
    const int k2 = lane & 15, h = lane >> 4;
#pragma unroll
    for (int m = 0; m < 16; m++) v[m] = tile[k2 * 33 + h + 2 * m];
    __syncwarp();
    dft16<S>(v);
    // radix-2 across lanes l, l^16: Z[k2 + 16 m + 256 b] = E0[m] +- w32^m E1[m]
#pragma unroll
    for (int m = 0; m < 16; m++) {
        double2 w = c_w32[m];
        if (S < 0) w.y = -w.y;
        v[m] = radix2_xlane(v[m], w, h);
    }
}

// ---------------------------------------------------------------------------
// Transforms of the lvl1 blind-rotation kernels.  The root table psi^t
// (t < N, psi = e^{i pi / N}; psi^{t+N} = -psi^t) lives in shared memory in
// the interleaved order pos(t) = (t mod 4) * 256 + t / 4, which makes the
// KeyBundle gathers psi^{(1+4f) a} (stride 4a across lanes) bank-conflict
// free for odd a.
__device__ __forceinline__ int psi_pos(uint32_t t) { return (int)((t & 3u) * 256u + ((t >> 2) & 255u)); }

// psi^t for any t (mod 2N)
__device__ __forceinline__ double2 psi_at(const double2* psi_s, uint32_t t)
{
    double2 v = psi_s[psi_pos(t)];
    if (t & 1024u) {
        v.x = -v.x;
        v.y = -v.y;
    }
    return v;
}

// e^{i pi n2 / 32} (= psi^{32 n2}, the compile-time part of the forward
// twist) and c_utwq[q] = e^{-i pi ((q mod 8) + 16 (q / 8)) / 64} times a
// power of two that each translation unit chooses (the compile-time part of
// the untwist of register q, with the inverse's normalisation and Torus
// scale folded in: 2^23 for N = 1024 Torus32, 2^54 for N = 2048 Torus64;
// power-of-two scaling commutes with every rounding)
static __constant__ double2 c_tw32[16];
static __constant__ double2 c_utwq[16];

// Where register q of `lane` lands after the lvl1 transforms: frequency bin
// (forward) or coefficient (inverse) k2 + 16 m + 256 b with k2 = lane & 15,
// m = (q & 7) + 8 (lane >> 4), b = q >> 3.
__device__ __forceinline__ int ffnt_pos(int lane, int q)
{
    return (lane & 15) + 16 * (q & 7) + 128 * (lane >> 4) + 256 * (q >> 3);
}

// -1 for first-stage lanes n1 = 3 (mod 4), else +1.  The second-stage lanes
// of the upper half (h = 1) read the first-stage lanes n1 = 1 + 2m, so with
// this sign folded into the first-stage twiddles their inputs arrive
// modulated by (-1)^m and their 16-point DFT comes out rotated by 8 bins,
// which lets both lanes of a radix-2 pair exchange the same registers.
__device__ __forceinline__ double lane_sign(int lane) { return (lane & 3) == 3 ? -1.0 : 1.0; }

// Radix-2 stage of the 32-point second stage across lanes l and l ^ 16, with
// every lane doing useful work.  On entry lanes h = 0 hold E0[q] in v[q] and
// lanes h = 1 hold E1[(q + 8) mod 16] (the lane_sign modulation).  Both send
// v[8 + j] to the partner, so that lane h holds E0[m] and E1[m] for
// m = j + 8 h; it writes E0 + w^m E1 to v[j] and E0 - w^m E1 to v[8 + j],
// w = e^{S 2 pi i / 32}.  Each output is rounded as in the textbook
// butterfly (t = w E1 rounded, then one add or subtract).
template <int S>
__device__ __forceinline__ void radix2_pair(double2 (&v)[16], int h)
{
#pragma unroll
    for (int j = 0; j < 8; j++) {
        double2 r;
        r.x = __shfl_xor_sync(0xffffffffu, v[8 + j].x, 16);
        r.y = __shfl_xor_sync(0xffffffffu, v[8 + j].y, 16);
        const double2 e0 = h ? r : v[j];
        const double2 e1 = h ? v[j] : r;
        double2 w = c_w32[j + 8 * h];
        if (S < 0) w.y = -w.y;
        const double2 t = cmul(e1, w);
        v[j] = cadd(e0, t);
        v[8 + j] = csub(e0, t);
    }
}

// Forward FFNT of one folded polynomial: in v[n2] = d[n] + i d[n + 512] for
// n = lane + 32 n2; out v[q] = bin ffnt_pos(lane, q).  (Storing the bins
// from inside the radix-2 stage keeps fewer registers live but measured
// slower.)  The twist
// psi^n = psi^lane psi^{32 n2} is split into a compile-time factor (before
// the 16-point DFT) and a per-lane factor merged with the w512^{lane k2}
// twiddle: lane_sign psi^{lane (1 + 4 k2)}, generated by recurrence from two
// table reads.
__device__ __forceinline__ void ffnt_forward_warp(double2 (&v)[16], double2* tile,
                                                  const double2* psi_s, int lane)
{
#pragma unroll
    for (int n2 = 1; n2 < 16; n2++) v[n2] = cmul(v[n2], c_tw32[n2]);
    dft16<1>(v);
    const double sg = lane_sign(lane);
    double2 t = psi_s[psi_pos((uint32_t)lane)];
    t.x *= sg;
    t.y *= sg;
    const double2 st = psi_s[psi_pos(4u * (uint32_t)lane)];
#pragma unroll
    for (int k2 = 0; k2 < 16; k2++) {
        v[k2] = cmul(v[k2], t);
        if (k2 < 15) t = cmul(t, st);
    }
#pragma unroll
    for (int k2 = 0; k2 < 16; k2++) tile[k2 * 33 + lane] = v[k2];
    __syncwarp();
    const int k2 = lane & 15, h = lane >> 4;
#pragma unroll
    for (int m = 0; m < 16; m++) v[m] = tile[k2 * 33 + h + 2 * m];
    __syncwarp();
    dft16<1>(v);
    radix2_pair<1>(v, h);
}

// Inverse FFNT: in v[n2] = Z[lane + 32 n2] (natural bins); out v[q] holds
// z'[n] conj(psi^n) 2^23 for n = ffnt_pos(lane, q): untwisted and in Torus32
// units before rounding (2^23 = 2^32 / 512).
__device__ __forceinline__ void ffnt_inverse_warp(double2 (&v)[16], double2* tile,
                                                  const double2* psi_s, int lane)
{
    dft16<-1>(v);
    {
        const double sg = lane_sign(lane);
        const double2 st = psi_s[psi_pos(4u * (uint32_t)lane)];  // w512^{lane} = psi^{4 lane}
        double2 t = make_double2(st.x * sg, st.y * sg);
        v[0].x *= sg;
        v[0].y *= sg;
#pragma unroll
        for (int k2 = 1; k2 < 16; k2++) {
            v[k2] = cmulc(v[k2], t);
            if (k2 < 15) t = cmul(t, st);
        }
    }
#pragma unroll
    for (int k2 = 0; k2 < 16; k2++) tile[k2 * 33 + lane] = v[k2];
    __syncwarp();
    const int k2 = lane & 15, h = lane >> 4;
#pragma unroll
    for (int m = 0; m < 16; m++) v[m] = tile[k2 * 33 + h + 2 * m];
    __syncwarp();
    dft16<-1>(v);
    radix2_pair<-1>(v, h);
    // untwist conj(psi^{k2 + 128 h}) conj(psi^{16 (q mod 8) + 256 (q / 8)}) 2^23
    const double2 u = psi_s[psi_pos((uint32_t)(k2 + 128 * h))];
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = cmul(cmulc(v[q], u), c_utwq[q]);
}

// ---------------------------------------------------------------------------
// Building blocks for N = 2048 (1024-point transform = two 512-point halves).
// A forward transform of the even (odd) samples z[2m (+1)], m = lane + 32 n2,
// whose twist psi2^{2m (+1)} = psi2^{2 lane (+1)} psi2^{64 n2} has the same
// compile-time factor c_tw32[n2] as the N = 1024 case; the per-lane factor
// t0 and the 512-point twiddle w512^{lane k2} = psi2^{8 lane k2} are merged
// into the geometric sequence t0 * step^k2 (with the lane_sign modulation of
// radix2_pair).  In: v[n2] already multiplied by c_tw32[n2].  Out: v[q] =
// bin ffnt_pos(lane, q) of the half.
__device__ __forceinline__ void dft512_fwd_post(double2 (&v)[16], double2* tile, int lane,
                                                double2 t, const double2 step)
{
    dft16<1>(v);
    const double sg = lane_sign(lane);
    t.x *= sg;
    t.y *= sg;
#pragma unroll
    for (int k2 = 0; k2 < 16; k2++) {
        v[k2] = cmul(v[k2], t);
        if (k2 < 15) t = cmul(t, step);
    }
#pragma unroll
    for (int k2 = 0; k2 < 16; k2++) tile[k2 * 33 + lane] = v[k2];
    __syncwarp();
    const int k2 = lane & 15, h = lane >> 4;
#pragma unroll
    for (int m = 0; m < 16; m++) v[m] = tile[k2 * 33 + h + 2 * m];
    __syncwarp();
    dft16<1>(v);
    radix2_pair<1>(v, h);
}

// Unscaled inverse 512-point DFT: in v[n2] = X[lane + 32 n2]; out v[q] =
// sum_k X[k] w512^{-n k} for n = ffnt_pos(lane, q).  wl = w512^{lane}.
__device__ __forceinline__ void dft512_inv_raw(double2 (&v)[16], double2* tile, int lane,
                                               const double2 wl)
{
    dft16<-1>(v);
    const double sg = lane_sign(lane);
    double2 t = make_double2(wl.x * sg, wl.y * sg);
    v[0].x *= sg;
    v[0].y *= sg;
#pragma unroll
    for (int k2 = 1; k2 < 16; k2++) {
        v[k2] = cmulc(v[k2], t);
        if (k2 < 15) t = cmul(t, wl);
    }
#pragma unroll
    for (int k2 = 0; k2 < 16; k2++) tile[k2 * 33 + lane] = v[k2];
    __syncwarp();
    const int k2 = lane & 15, h = lane >> 4;
#pragma unroll
    for (int m = 0; m < 16; m++) v[m] = tile[k2 * 33 + h + 2 * m];
    __syncwarp();
    dft16<-1>(v);
    radix2_pair<-1>(v, h);
}

}  // namespace cufhe
