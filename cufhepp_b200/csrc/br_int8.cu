// Exact INT8 tensor-core blind rotation (tcgen05, sm_100a), plain CMUX form.
//
// Step i of __BlindRotate__ (include/gatebootstrapping_gpu.cuh:801-884) is
//   acc += ExtProd(BK_i, X^abar acc - acc),
// i.e. for every lane (gate) and output polynomial j_out
//   out[j_out][n] = sum_{r, m} dec_r[m] * sign(n, m) * BK_i[r][j_out][(n - m) mod N]
// with signed gadget digits dec_r in [-128, 128) (l = 2, Bgbit = 8, r = j*2 + d).
// This is a GEMM whose shared operand is the negacyclic Toeplitz expansion of
// the key: rows (j_out, n), columns (r, m), M = 2048 rows per limb, K = 4096.
//
// Exactness.  Each key word is split into four balanced signed byte limbs
// (v = sum_c s_c 2^(8c) mod 2^32, s_c in [-128, 128)); digits are s8 as well,
// so kind::i8 products are exact and a K = 4096 sum is bounded by
// 4096 * 128 * 128 = 2^26 in INT32.  The epilogue recombines
// sum_c acc_c << (8c) mod 2^32, which is the exact Torus32 result: the
// blind rotation is bit-identical to the schoolbook oracle.
//
// Layout.
//  * key  : for step i, output poly j, row r, limb c a 2N-byte sequence
//           V[t] = limb_c(BK[N-1-t]) (t < N), limb_c(-BK[2N-1-t]) (t >= N),
//           so Toeplitz row n restricted to columns [m0, m0+128) is the
//           contiguous window V[N-1-n+m0 .. +128): negacyclic signs are
//           folded into the table, nothing is negated at run time.
//           [636][2][4][4][2048] int8 = 41.7 MB.
//  * digits: per group of 256 lanes and K chunk of 128, a 32 KB tile already in
//           the canonical K-major 128B-swizzled shared-memory layout, moved by
//           cp.async.bulk (one contiguous copy per chunk).
//  * acc  : [lanes][2][1024] Torus32.
//
// k_i8_gemm_p (one launch per step, one CTA per SM): tile = (256-lane group,
// 128 output rows = 4 limbs x 32 coefficients of one j_out), warp-specialised:
// two generator warpgroups write the Toeplitz A chunks straight into TMEM
// (tcgen05.st; thread = row), one thread issues 4 tcgen05.mma.kind::i8
// (M=128, N=256, K=32) per chunk into the INT32 accumulator in TMEM, two
// threads stream the digit chunks through a 5-stage shared-memory ring, and
// sixteen drain warps fold the limbs and add them into the global
// accumulator.  Hand-offs go through mbarriers only; every wait is bounded
// and reports a timeout through an error flag instead of hanging.
#include <stdio.h>
#include <stdlib.h>

#include <atomic>

#include <cuda.h>

#include "br_int8.h"
#include "engine.h"
#include "tc_util.cuh"

namespace cufhe {

namespace {

constexpr int kGroup = 256;                  // lanes per MMA N
constexpr int kChunkK = 128;                 // K bytes per chunk (one swizzle row)
constexpr int kChunks = 4 * kN / kChunkK;    // 32
constexpr int kTileBytes = kGroup * kChunkK; // 32 KB
constexpr int kRowsCoef = 32;                // coefficients per CTA tile (x4 limbs = 128 rows)
constexpr int kVBytesStep = 2 * 4 * 4 * 2 * kN;  // 64 KB of key table per step
constexpr int kVBytesJ = 4 * 4 * 2 * kN;         // 32 KB per output poly
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kAccCol = 0;      // accumulator columns [0, 256)
constexpr uint32_t kACol = 256;      // A slots: 32 columns each from column 256

// instruction descriptor: D s32, A s8, B s8, K-major both, N = 256, M = 128
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kGroup >> 3) << 17) |
                            ((uint32_t)(128 >> 4) << 24);

// ------------------------------------------------------------ kernels ----

// key table: out[i][j][r][c][t], t < 2N (4 bytes per thread), i over the
// key's ntrgsw TRGSWs (636 plain, 318 x 3 KeyBundle)
__global__ void k_i8_key(const uint32_t* __restrict__ bk, int ntrgsw, int8_t* __restrict__ out)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // 4-byte unit
    const size_t total = (size_t)ntrgsw * kVBytesStep / 4;
    if (q >= total) return;
    const size_t byte = q * 4;
    const int t0 = (int)(byte % (2 * kN));
    size_t rest = byte / (2 * kN);
    const int c = (int)(rest % 4);
    rest /= 4;
    const int r = (int)(rest % 4);
    rest /= 4;
    const int j = (int)(rest % 2);
    const size_t i = rest / 2;
    const uint32_t* poly = bk + ((i * 4 + r) * 2 + j) * kN;  // TFHEpp TRGSW[i][r][j][N]
    uint32_t packed = 0;
    for (int e = 0; e < 4; e++) {
        const int t = t0 + e;
        const uint32_t x = t < kN ? poly[kN - 1 - t] : 0u - poly[2 * kN - 1 - t];
        packed |= (uint32_t)(uint8_t)limb(x, c) << (8 * e);
    }
    reinterpret_cast<uint32_t*>(out)[q] = packed;
}

// modulus switch + test vector (RotatedTestVector, bar unrounded, abar rounded)
__global__ void k_i8_init(const uint32_t* __restrict__ lane_in, int lanes, uint32_t mu,
                          uint16_t* __restrict__ abar, uint32_t* __restrict__ acc)
{
    const int l = blockIdx.x;
    if (l >= lanes) return;
    const uint32_t* x = lane_in + (size_t)l * kTlwe0;
    for (int i = threadIdx.x; i < kN0; i += blockDim.x)
        abar[(size_t)l * 640 + i] = (uint16_t)((x[i] + (1u << 20)) >> 21);
    const uint32_t bar = 2u * kN - (x[kN0] >> 21);
    uint32_t* a = acc + (size_t)l * kTrlwe;
    for (int i = threadIdx.x; i < kN; i += blockDim.x) {
        a[i] = 0;
        a[kN + i] = bar == 2u * kN ? mu
                                    : ((((uint32_t)i < (bar & (kN - 1))) ^ (bar >> 10)) ? 0u - mu : mu);
    }
}

// Digits of the step's external-product input, written as swizzled tiles
// tiles[group][chunk][32 KB]; one CTA (256 threads) per lane, 4 coefficients
// per thread and polynomial.
//  * plain CMUX step `step`: digits of X^abar acc - acc (acc is only read);
//  * KeyBundle pair (KB): digits of acc itself, and acc is overwritten in
//    place with their gadget recomposition sum_d dec_d 2^(32 - 8 (d + 1)) =
//    (acc + 2^15) & 0xFFFF0000 -- the H term of the combined key
//    H + sum_j bk_j (X^(e_j) - 1), to which the pair's GEMM then adds the
//    rotated products (include/gatebootstrapping_gpu.cuh:928-948, :966-994).
//    Each thread reads and rewrites only its own coefficients.
template <bool KB>
__global__ void __launch_bounds__(256) k_i8_decompose(uint32_t* __restrict__ acc,
                                                      const uint16_t* __restrict__ abar, int lanes,
                                                      int step, uint8_t* __restrict__ tiles)
{
    // launched as a programmatic dependent of the previous step's GEMM: wait
    // for its accumulator updates before reading the accumulator
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int l = blockIdx.x;
    if (l >= lanes) return;
    const uint32_t row = (uint32_t)(l % kGroup);
    uint8_t* gtile = tiles + (size_t)(l / kGroup) * kChunks * kTileBytes;
    const int m = threadIdx.x * 4;
    constexpr uint32_t kOff = (128u << 24) + (128u << 16) + (1u << 15);
    uint32_t ab = 0, abm = 0, abn = 0, base = 0, q0 = 0, off = 0;
    if (!KB) {
        ab = abar[(size_t)l * 640 + step];
        abm = ab & (kN - 1);
        abn = ab >> 10;
        // the rotated window a[(m - ab) ..  + 4) from two aligned 16-byte loads
        base = ((uint32_t)m - ab) & (kN - 1);
        q0 = base & ~3u;
        off = base & 3u;
    }
#pragma unroll
    for (int j = 0; j < 2; j++) {
        uint32_t* a = acc + (size_t)l * kTrlwe + j * kN;
        const uint4 cur = *reinterpret_cast<const uint4*>(a + m);
        const uint32_t cv[4] = {cur.x, cur.y, cur.z, cur.w};
        uint32_t x[4];
        if (KB) {
#pragma unroll
            for (int e = 0; e < 4; e++) x[e] = cv[e];
            *reinterpret_cast<uint4*>(a + m) =
                make_uint4((cv[0] + (1u << 15)) & 0xFFFF0000u, (cv[1] + (1u << 15)) & 0xFFFF0000u,
                           (cv[2] + (1u << 15)) & 0xFFFF0000u, (cv[3] + (1u << 15)) & 0xFFFF0000u);
        } else {
            const uint4 w0 = *reinterpret_cast<const uint4*>(a + q0);
            const uint4 w1 = *reinterpret_cast<const uint4*>(a + ((q0 + 4) & (kN - 1)));
            const uint32_t win[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const uint32_t n = (uint32_t)(m + e);
                // win[off + e] without a dynamic register index
                uint32_t rv = off == 0 ? win[e] : off == 1 ? win[e + 1] : off == 2 ? win[e + 2] : win[e + 3];
                rv = ((n < abm) ^ abn) ? 0u - rv : rv;
                x[e] = rv - cv[e];
            }
        }
        uint32_t d0 = 0, d1 = 0;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const uint32_t t = x[e] + kOff;
            d0 |= (uint32_t)(uint8_t)((int)((t >> 24) & 255u) - 128) << (8 * e);
            d1 |= (uint32_t)(uint8_t)((int)((t >> 16) & 255u) - 128) << (8 * e);
        }
#pragma unroll
        for (int d = 0; d < 2; d++) {
            const uint32_t K = (uint32_t)((2 * j + d) * kN + m);
            uint8_t* t = gtile + (size_t)(K / kChunkK) * kTileBytes + swz_offset(row, K % kChunkK);
            *reinterpret_cast<uint32_t*>(t) = d ? d1 : d0;
        }
    }
}

// ---- persistent form of the step GEMM -------------------------------------
// One CTA per SM; CTA b serves output polynomial j = b & 1 and walks that
// polynomial's tiles t = b >> 1, + gridDim.x / 2, ... (tile = 256-lane digit
// group x 128 rows = 4 limbs x 32 coefficients), so it keeps one 32 KB key
// window, TMEM and the barriers for its whole life.  The tiles of the last,
// partial round are split along K (unit_of), so a batch whose tile count is
// not a multiple of the CTA count ends with a fraction of a tile, not a whole
// one; the drain adds every unit into the global accumulator atomically.  Each K chunk has ONE
// full barrier (the producer's transaction bytes and the 128 A-generator
// arrivals) and ONE empty barrier (the MMA commit): with one wait and one
// commit per chunk the issuing thread keeps up with M128 N256 K32 MMAs.
// Roles:
//   warps 0-7   generators: Toeplitz A chunks into five 32-column TMEM slots
//               (chunk g uses slot g mod 5; warpgroup g mod 2 writes it)
//   warp 8      MMA issue: 4 x tcgen05.mma.kind::i8 M128 N256 K32 per chunk
//   warps 9, 26 producers: the key window once (warp 9), then 32 KB digit
//               chunks through a 5-stage ring across all tiles, even chunks
//               from warp 9 and odd chunks from warp 26 (one issuing thread
//               sustains about one bulk copy per 800 cycles, two keep the
//               ring ahead of the MMAs)
//   warps 10-25 drainers (four per TMEM lane quadrant, 64 columns each):
//               read the accumulator, add the four limb rows into a shared
//               [256 lanes][32 coefficients] buffer (limb q shifted by 8q),
//               release the accumulator, then add the buffer atomically into
//               the global accumulator while the next unit's MMAs run
// Every wait is bounded; an expired wait sets s_fail, which all roles poll.
constexpr int kPStages = 5;
constexpr size_t kSmemPB = (size_t)kPStages * kTileBytes;                // 160 KB
constexpr size_t kSmemPV = kVBytesJ;                                      // 32 KB
constexpr size_t kRedWords = (size_t)kGroup * kRowsCoef;                  // 8192
constexpr size_t kSmemPRed = kRedWords * 4;                               // 32 KB
constexpr size_t kSmemGemmP = 1024 + kSmemPB + kSmemPV + kSmemPRed + 512;
constexpr int kDrainWarps = 16;
constexpr int kGemmPThreads = 32 * (11 + kDrainWarps);                    // 864

// 32 lanes x 16 columns x 32 bit
__device__ __forceinline__ void tmem_st16(uint32_t addr, const uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16};"
        ::"r"(addr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]),
          "r"(v[7]), "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]),
          "r"(v[14]), "r"(v[15])
        : "memory");
}

// Work unit `it` of CTA cb: the first R units are whole tiles
// t = cb + it * ncj (all 32 K chunks); the tiles of the last, partial round
// are split along K into `split` units of 32 / split chunks each, dealt out
// over the CTAs, so that the last round costs 1 / split of a tile.
__device__ __forceinline__ void unit_of(int it, const int* geo, int& t, int& k0, int& nk)
{
    // geo = {R, cb, ncj, split}
    const int R = geo[0], cb = geo[1], ncj = geo[2];
    if (it < R) {
        t = cb + it * ncj;
        k0 = 0;
        nk = kChunks;
    } else {
        const int split = geo[3], u = cb + (it - R) * ncj;
        t = R * ncj + u / split;
        nk = kChunks / split;
        k0 = (u % split) * nk;
    }
}

template <bool KB>
__global__ void __launch_bounds__(kGemmPThreads, 1) k_i8_gemm_p(const int8_t* __restrict__ vkey,
                                                                const uint8_t* __restrict__ tiles,
                                                                uint32_t* __restrict__ acc,
                                                                int lanes, int tiles_j, int split,
                                                                const uint16_t* __restrict__ abar,
                                                                int pair, int* __restrict__ err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t raw_addr = smem_u32(smem_raw);
    unsigned char* smem = smem_raw + ((1024u - (raw_addr & 1023u)) & 1023u);
    unsigned char* bst = smem;
    int8_t* vs = reinterpret_cast<int8_t*>(smem + kSmemPB);
    uint32_t* red = reinterpret_cast<uint32_t*>(smem + kSmemPB + kSmemPV);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kSmemPB + kSmemPV + kSmemPRed);
    uint64_t* full = bars;                    // [kPStages]
    uint64_t* empty = full + kPStages;        // [kPStages]
    uint64_t* acc_full = empty + kPStages;
    uint64_t* acc_empty = acc_full + 1;
    uint64_t* bar_v = acc_empty + 1;
    uint64_t* red_full = bar_v + 1;
    uint64_t* red_clear = red_full + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(red_clear + 1);
    __shared__ volatile int s_fail;
    __shared__ int s_geo[5];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // combo = key * 2 + j_out: the plain form has one key per step, the
    // KeyBundle form three (bk0, bk1, bk2 of the pair)
    constexpr int kCombos = KB ? 6 : 2;
    const int combo = (int)(blockIdx.x % kCombos), j_out = combo & 1;
    const int cb = (int)(blockIdx.x / kCombos), ncj = (int)(gridDim.x / kCombos);
    const int R = tiles_j / ncj, NU = (tiles_j - R * ncj) * split;
    const int T = R + (cb < NU ? (NU - 1 - cb) / ncj + 1 : 0);

    for (size_t i = tid; i < kRedWords; i += blockDim.x) red[i] = 0u;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        s_fail = 0;
        s_geo[0] = R;
        s_geo[1] = cb;
        s_geo[2] = ncj;
        s_geo[3] = split;
        s_geo[4] = combo;
        for (int s = 0; s < kPStages; s++) {
            mbar_init(&full[s], 128 + 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, kDrainWarps);
        mbar_init(bar_v, 1);
        mbar_init(red_full, kDrainWarps);
        mbar_init(red_clear, kDrainWarps);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 9 || warp == 10 + kDrainWarps) {
        // ---- producers: warp 9 even chunks, the last warp odd chunks
        const int par = warp == 9 ? 0 : 1;
        if (lane == 0) {
            if (par == 0) {
                mbar_expect_tx(bar_v, (uint32_t)kSmemPV);
                bulk_g2s(vs, vkey + (size_t)combo * kVBytesJ, (uint32_t)kSmemPV, bar_v);
            }
            // the key window above is constant; the digit tiles are the
            // previous kernel's output (programmatic dependent launch)
            asm volatile("griddepcontrol.wait;" ::: "memory");
            int gbase = 0;
            for (int it = 0; it < T && !s_fail; it++) {
                int t, k0, nk;
                unit_of(it, s_geo, t, k0, nk);
                const int group = t / (kN / kRowsCoef);
                const uint8_t* gt = tiles + (size_t)group * kChunks * kTileBytes;
                for (int lk = par; lk < nk; lk += 2) {
                    const int kc = k0 + lk, gc = gbase + lk, s = gc % kPStages;
                    if (s_fail) break;
                    if (gc >= kPStages &&
                        !mbar_wait(&empty[s], (uint32_t)((gc / kPStages) - 1) & 1)) {
                        s_fail = 1;
                        break;
                    }
                    mbar_expect_tx(&full[s], kTileBytes);
                    bulk_g2s(bst + s * kTileBytes, gt + (size_t)kc * kTileBytes, kTileBytes, &full[s]);
                }
                gbase += nk;
            }
        }
    } else if (warp == 8) {
        // ---- MMA issue
        if (lane == 0) {
            int gc = 0;
            for (int it = 0; it < T && !s_fail; it++) {
                int t, k0, nk;
                unit_of(it, s_geo, t, k0, nk);
                if (it >= 1 && !mbar_wait(acc_empty, (uint32_t)(it - 1) & 1)) {
                    s_fail = 1;
                    break;
                }
                tc_fence_after();
                for (int lk = 0; lk < nk; lk++, gc++) {
                    const int s = gc % kPStages;
                    if (!mbar_wait(&full[s], (uint32_t)(gc / kPStages) & 1)) {
                        s_fail = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t bbase = smem_u32(bst + s * kTileBytes);
#pragma unroll
                    for (int k = 0; k < kChunkK / 32; k++)
                        tc_mma_i8(tmem + kAccCol, tmem + kACol + 32 * s + 8 * k,
                                  desc_kmajor_sw128(bbase + 32 * k), kIdesc, (lk | k) != 0);
                    tc_commit(&empty[s]);
                }
                if (s_fail) break;
                tc_commit(acc_full);
            }
        }
    } else if (warp < 8) {
        // ---- generators: warpgroup wg writes the chunks of parity wg
        const int wg = warp >> 2, q = warp & 3;
        const uint32_t lane_base = (uint32_t)(32 * q) << 16;
        bool ok = __all_sync(0xffffffffu, mbar_wait(bar_v, 0));
        int gbase = 0;
        for (int it = 0; it < T && ok; it++) {
            int t, k0, nk;
            unit_of(it, s_geo, t, k0, nk);
            const int n = (t % (kN / kRowsCoef)) * kRowsCoef + lane;
            for (int lk = wg; lk < nk; lk += 2) {
                const int kc = k0 + lk, gc = gbase + lk, s = gc % kPStages;
                if (__any_sync(0xffffffffu, s_fail != 0)) {
                    ok = false;
                    break;
                }
                if (gc >= kPStages &&
                    !__all_sync(0xffffffffu,
                                mbar_wait(&empty[s], (uint32_t)((gc / kPStages) - 1) & 1))) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const int r = kc / (kN / kChunkK), m0 = (kc % (kN / kChunkK)) * kChunkK;
                const uint32_t* vw =
                    reinterpret_cast<const uint32_t*>(vs + (size_t)(r * 4 + q) * (2 * kN));
                const int sst = kN - 1 - n + m0;
                const int w0 = sst >> 2, sh = (sst & 3) * 8;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    uint32_t w[17];
#pragma unroll
                    for (int i = 0; i < 17; i++) w[i] = vw[w0 + 16 * h + i];
                    uint32_t a[16];
#pragma unroll
                    for (int i = 0; i < 16; i++) a[i] = __funnelshift_r(w[i], w[i + 1], sh);
                    tmem_st16(tmem + lane_base + kACol + 32 * s + 16 * h, a);
                }
                tmem_wait_st();
                tc_fence_before();
                mbar_arrive(&full[s]);
            }
            gbase += nk;
        }
        if (!ok) s_fail = 1;
    } else {
        // ---- drainers: warp d reads TMEM lane quadrant warp % 4 (the hardware
        // ties a warp to quadrant warp % 4), accumulator columns [64 p, 64 p + 64)
        const int d = warp - 10, q = warp & 3, p = d >> 2;
        const uint32_t lane_base = (uint32_t)(32 * q) << 16;
        asm volatile("griddepcontrol.wait;" ::: "memory");
        bool ok = true;
        for (int it = 0; it < T && ok; it++) {
            if (__any_sync(0xffffffffu, s_fail != 0) ||
                !__all_sync(0xffffffffu, mbar_wait(acc_full, (uint32_t)it & 1))) {
                ok = false;
                break;
            }
            tc_fence_after();
            // both column blocks into registers first: the accumulator is
            // released before the shared-buffer adds, so the next tile's MMAs
            // wait only for the TMEM reads
            uint32_t v0[32], v1[32];
            tmem_ld32(tmem + lane_base + kAccCol + 64 * p, v0);
            tmem_ld32(tmem + lane_base + kAccCol + 64 * p + 32, v1);
            tmem_wait_ld();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(acc_empty);
#pragma unroll
            for (int i = 0; i < 32; i++)
                atomicAdd(&red[(size_t)(64 * p + i) * kRowsCoef + lane], v0[i] << (8 * q));
#pragma unroll
            for (int i = 0; i < 32; i++)
                atomicAdd(&red[(size_t)(64 * p + 32 + i) * kRowsCoef + lane], v1[i] << (8 * q));
            __threadfence_block();  // this warp's shared-buffer adds before the hand-off
            __syncwarp();
            if (lane == 0) mbar_arrive(red_full);
            if (!__all_sync(0xffffffffu, mbar_wait(red_full, (uint32_t)it & 1))) {
                ok = false;
                break;
            }
            int t, k0, nk;
            unit_of(it, s_geo, t, k0, nk);
            const int group = t / (kN / kRowsCoef);
            const int n0 = (t % (kN / kRowsCoef)) * kRowsCoef;
            constexpr int kW = kGroup / kDrainWarps;
            // a tile split along K is added by several CTAs, and in the
            // KeyBundle form three keys add into every word: atomic adds (mod
            // 2^32, so their order does not matter)
            if (KB) {
                // P = Dec(acc) . bk_key enters as (X^e - 1) P, with
                // e = a0 + a1, a0, a1 for bk0, bk1, bk2
                const int key = s_geo[4] >> 1;
                const uint32_t n = (uint32_t)(n0 + lane);
                // the kW gate lanes' rotation pairs (a0, a1 in one 32-bit word),
                // loaded together and then broadcast, not one dependent load
                // per iteration
                uint32_t my_a01 = 0;
                {
                    const int l = group * kGroup + d + kDrainWarps * lane;
                    if (lane < kW && l < lanes)
                        my_a01 = *reinterpret_cast<const uint32_t*>(abar + (size_t)l * 640 + 2 * pair);
                }
#pragma unroll 1
                for (int i = 0; i < kW; i++) {
                    const int gl = d + kDrainWarps * i, l = group * kGroup + gl;
                    const uint32_t v = red[(size_t)gl * kRowsCoef + lane];
                    red[(size_t)gl * kRowsCoef + lane] = 0u;
                    const uint32_t a01 = __shfl_sync(0xffffffffu, my_a01, i);
                    if (l < lanes) {
                        const uint32_t a0 = a01 & 0xFFFFu, a1 = a01 >> 16;
                        const uint32_t e = key == 0 ? (a0 + a1) & (2 * kN - 1) : key == 1 ? a0 : a1;
                        const uint32_t pos = (n + e) & (2 * kN - 1);
                        uint32_t* out = acc + (size_t)l * kTrlwe + j_out * kN;
                        atomicAdd(&out[pos & (kN - 1)], pos < (uint32_t)kN ? v : 0u - v);
                        atomicAdd(&out[n], 0u - v);
                    }
                }
            } else {
#pragma unroll
                for (int i = 0; i < kW; i++) {
                    const int gl = d + kDrainWarps * i, l = group * kGroup + gl;
                    const uint32_t v = red[(size_t)gl * kRowsCoef + lane];
                    red[(size_t)gl * kRowsCoef + lane] = 0u;
                    if (l < lanes) atomicAdd(&acc[(size_t)l * kTrlwe + j_out * kN + n0 + lane], v);
                }
            }
            __threadfence_block();  // the zeroed buffer before the next tile's adds
            __syncwarp();
            if (lane == 0) mbar_arrive(red_clear);
            if (!__all_sync(0xffffffffu, mbar_wait(red_clear, (uint32_t)it & 1))) {
                ok = false;
                break;
            }
        }
        if (!ok) s_fail = 1;
    }

    __syncthreads();
    if (s_fail && tid == 0) {
        atomicOr(err, 1);
        // drain: wait (bounded) for copies and MMA batches that may be in flight
        for (int s = 0; s < kPStages; s++) mbar_wait(&full[s], 0), mbar_wait(&full[s], 1);
        mbar_wait(acc_full, 0), mbar_wait(acc_full, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols));
}

// ---- CTA-pair form of the step GEMM (tcgen05 cta_group::2) ----------------
// A cluster of two CTAs on two SMs shares every digit tile: each CTA copies
// its half of the tile's 256 lanes (16 KB per chunk instead of 32) and
// generates the Toeplitz A rows of its own (key, output polynomial) combo,
// and the even CTA issues M = 256 MMAs (128 rows in each CTA's TMEM, lanes
// split between the two CTAs' shared memory) for both.  Each SM therefore
// moves half the digit bytes and issues half the MMAs of k_i8_gemm_p for the
// same work.  Rank r of a pair serves output polynomial r; pair type
// (KeyBundle: the key of the pair) = cluster mod kPairTypes.
//   warps 0-7   generators (own combo), as in k_i8_gemm_p
//   warp 8      even CTA: MMA issue for the pair; its chunk barrier counts
//               both CTAs' digit bytes (the odd CTA's tensor copies complete
//               on it) and both CTAs' generators (the odd CTA's warps arrive
//               remotely), and the odd CTA's drain warps release the
//               accumulator remotely; every MMA batch commits to the
//               barriers of both CTAs
//   warps 9, 26 producers: own half of each digit chunk, own key window
//   warps 10-25 drainers (own 128 rows of the accumulator), as in k_i8_gemm_p
// Every wait is bounded; both CTAs always meet at the closing cluster barrier
// before the pair releases its TMEM.
constexpr int kHalfTile = kTileBytes / 2;                                  // 16 KB
// digit ring depth of the pair form (half chunks; A slots: 32 TMEM columns
// each from column 256).  Measured at 4789 lanes, KeyBundle: 5 stages
// 116.5 ms per rotation, 6 stages 115.1 ms, 8 stages 116.5 ms.
constexpr int kPairStages = 6;
constexpr size_t kSmemPairB = (size_t)kPairStages * kHalfTile;
constexpr size_t kSmemGemmPair = 1024 + kSmemPairB + kSmemPV + kSmemPRed + 512;
constexpr uint32_t kIdescPair = idesc_i8(256, kGroup);

template <bool KB>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kGemmPThreads, 1)
    k_i8_gemm_2sm(const __grid_constant__ CUtensorMap tmap, const int8_t* __restrict__ vkey,
                  const uint8_t* __restrict__ tiles,
                  uint32_t* __restrict__ acc, int lanes, int tiles_j, int split,
                  const uint16_t* __restrict__ abar, int pair, int* __restrict__ err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t raw_addr = smem_u32(smem_raw);
    unsigned char* smem = smem_raw + ((1024u - (raw_addr & 1023u)) & 1023u);
    unsigned char* bst = smem;
    int8_t* vs = reinterpret_cast<int8_t*>(smem + kSmemPairB);
    uint32_t* red = reinterpret_cast<uint32_t*>(smem + kSmemPairB + kSmemPV);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kSmemPairB + kSmemPV + kSmemPRed);
    uint64_t* full = bars;                    // [kPairStages]
    uint64_t* empty = full + kPairStages;        // [kPairStages]
    uint64_t* acc_full = empty + kPairStages;
    uint64_t* acc_empty = acc_full + 1;
    uint64_t* bar_v = acc_empty + 1;
    uint64_t* red_full = bar_v + 1;
    uint64_t* red_clear = red_full + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(red_clear + 1);
    __shared__ volatile int s_fail;
    __shared__ int s_geo[5];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = cluster_rank();
    constexpr int kPairTypes = KB ? 3 : 1;
    const int q = (int)(blockIdx.x >> 1);
    const int combo = (q % kPairTypes) * 2 + (int)rank, j_out = (int)rank;
    const int cb = q / kPairTypes, ncj = (int)(gridDim.x >> 1) / kPairTypes;
    const int R = tiles_j / ncj, NU = (tiles_j - R * ncj) * split;
    const int T = R + (cb < NU ? (NU - 1 - cb) / ncj + 1 : 0);

    for (size_t i = tid; i < kRedWords; i += blockDim.x) red[i] = 0u;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    if (tid == 0) {
        s_fail = 0;
        s_geo[0] = R;
        s_geo[1] = cb;
        s_geo[2] = ncj;
        s_geo[3] = split;
        s_geo[4] = combo;
        for (int s = 0; s < kPairStages; s++) {
            // (even CTA) 128 own generator threads, its producer, 4 odd generator warps
            mbar_init(&full[s], 128 + 1 + 4);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, 2 * kDrainWarps);  // (even CTA) both CTAs' drain warps
        mbar_init(bar_v, 1);
        mbar_init(red_full, kDrainWarps);
        mbar_init(red_clear, kDrainWarps);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();  // both CTAs' barriers exist before any remote arrival
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 9 || warp == 10 + kDrainWarps) {
        // ---- producers: this CTA's half (lanes 128 r ..) of each digit chunk
        const int par = warp == 9 ? 0 : 1;
        if (lane == 0) {
            if (par == 0) {
                mbar_expect_tx(bar_v, (uint32_t)kSmemPV);
                bulk_g2s(vs, vkey + (size_t)combo * kVBytesJ, (uint32_t)kSmemPV, bar_v);
            }
            asm volatile("griddepcontrol.wait;" ::: "memory");
            int gbase = 0;
            for (int it = 0; it < T && !s_fail; it++) {
                int t, k0, nk;
                unit_of(it, s_geo, t, k0, nk);
                const int group = t / (kN / kRowsCoef);
                const uint8_t* gt = tiles + (size_t)group * kChunks * kTileBytes;
                for (int lk = par; lk < nk; lk += 2) {
                    const int kc = k0 + lk, gc = gbase + lk, s = gc % kPairStages;
                    if (s_fail) break;
                    if (gc >= kPairStages &&
                        !mbar_wait(&empty[s], (uint32_t)((gc / kPairStages) - 1) & 1)) {
                        s_fail = 1;
                        break;
                    }
                    if (rank == 0) {
                        // both halves' bytes land on this barrier
                        mbar_expect_tx(&full[s], kTileBytes);
                        bulk_g2s(bst + s * kHalfTile, gt + (size_t)kc * kTileBytes, kHalfTile,
                                 &full[s]);
                    } else {
                        // rows 128..255 of chunk kc of the group, as 128 rows x 128 B
                        tma2d_g2s_to_even(bst + s * kHalfTile, &tmap, 0,
                                          (group * kChunks + kc) * kGroup + 128, &full[s]);
                    }
                }
                gbase += nk;
            }
        }
    } else if (warp == 8) {
        if (lane == 0 && rank == 0) {
            // ---- MMA issue for the pair
            int gc = 0;
            for (int it = 0; it < T && !s_fail; it++) {
                int t, k0, nk;
                unit_of(it, s_geo, t, k0, nk);
                if (it >= 1 && !mbar_wait(acc_empty, (uint32_t)(it - 1) & 1)) {
                    s_fail = 1;
                    break;
                }
                tc_fence_after();
                for (int lk = 0; lk < nk; lk++, gc++) {
                    const int s = gc % kPairStages;
                    if (!mbar_wait(&full[s], (uint32_t)(gc / kPairStages) & 1)) {
                        s_fail = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t bbase = smem_u32(bst + s * kHalfTile);
#pragma unroll
                    for (int k = 0; k < kChunkK / 32; k++)
                        tc_mma_i8_pair(tmem + kAccCol, tmem + kACol + 32 * s + 8 * k,
                                       desc_kmajor_sw128(bbase + 32 * k), kIdescPair, (lk | k) != 0);
                    tc_commit_pair(&empty[s]);
                }
                if (s_fail) break;
                tc_commit_pair(acc_full);
            }
        }
    } else if (warp < 8) {
        // ---- generators: this CTA's combo, chunks of parity wg
        const int wg = warp >> 2, qd = warp & 3;
        const uint32_t lane_base = (uint32_t)(32 * qd) << 16;
        bool ok = __all_sync(0xffffffffu, mbar_wait(bar_v, 0));
        int gbase = 0;
        for (int it = 0; it < T && ok; it++) {
            int t, k0, nk;
            unit_of(it, s_geo, t, k0, nk);
            const int n = (t % (kN / kRowsCoef)) * kRowsCoef + lane;
            for (int lk = wg; lk < nk; lk += 2) {
                const int kc = k0 + lk, gc = gbase + lk, s = gc % kPairStages;
                if (__any_sync(0xffffffffu, s_fail != 0)) {
                    ok = false;
                    break;
                }
                if (gc >= kPairStages &&
                    !__all_sync(0xffffffffu,
                                mbar_wait(&empty[s], (uint32_t)((gc / kPairStages) - 1) & 1))) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const int r = kc / (kN / kChunkK), m0 = (kc % (kN / kChunkK)) * kChunkK;
                const uint32_t* vw =
                    reinterpret_cast<const uint32_t*>(vs + (size_t)(r * 4 + qd) * (2 * kN));
                const int sst = kN - 1 - n + m0;
                const int w0 = sst >> 2, sh = (sst & 3) * 8;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    uint32_t w[17];
#pragma unroll
                    for (int i = 0; i < 17; i++) w[i] = vw[w0 + 16 * h + i];
                    uint32_t a[16];
#pragma unroll
                    for (int i = 0; i < 16; i++) a[i] = __funnelshift_r(w[i], w[i + 1], sh);
                    tmem_st16(tmem + lane_base + kACol + 32 * s + 16 * h, a);
                }
                tmem_wait_st();
                tc_fence_before();
                if (rank == 0) {
                    mbar_arrive(&full[s]);
                } else {
                    __syncwarp();
                    if (lane == 0) mbar_arrive_cluster(&full[s], 0);
                }
            }
            gbase += nk;
        }
        if (!ok) s_fail = 1;
    } else {
        // ---- drainers: this CTA's 128 rows (its combo), all 256 lanes
        const int d = warp - 10, qd = warp & 3, pq = d >> 2;
        const uint32_t lane_base = (uint32_t)(32 * qd) << 16;
        asm volatile("griddepcontrol.wait;" ::: "memory");
        bool ok = true;
        for (int it = 0; it < T && ok; it++) {
            if (__any_sync(0xffffffffu, s_fail != 0) ||
                !__all_sync(0xffffffffu, mbar_wait(acc_full, (uint32_t)it & 1))) {
                ok = false;
                break;
            }
            tc_fence_after();
            uint32_t v0[32], v1[32];
            tmem_ld32(tmem + lane_base + kAccCol + 64 * pq, v0);
            tmem_ld32(tmem + lane_base + kAccCol + 64 * pq + 32, v1);
            tmem_wait_ld();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                if (rank == 0)
                    mbar_arrive(acc_empty);
                else
                    mbar_arrive_cluster(acc_empty, 0);
            }
#pragma unroll
            for (int i = 0; i < 32; i++)
                atomicAdd(&red[(size_t)(64 * pq + i) * kRowsCoef + lane], v0[i] << (8 * qd));
#pragma unroll
            for (int i = 0; i < 32; i++)
                atomicAdd(&red[(size_t)(64 * pq + 32 + i) * kRowsCoef + lane], v1[i] << (8 * qd));
            __threadfence_block();
            __syncwarp();
            if (lane == 0) mbar_arrive(red_full);
            if (!__all_sync(0xffffffffu, mbar_wait(red_full, (uint32_t)it & 1))) {
                ok = false;
                break;
            }
            int t, k0, nk;
            unit_of(it, s_geo, t, k0, nk);
            const int group = t / (kN / kRowsCoef);
            const int n0 = (t % (kN / kRowsCoef)) * kRowsCoef;
            constexpr int kW = kGroup / kDrainWarps;
            if (KB) {
                const int key = s_geo[4] >> 1;
                const uint32_t n = (uint32_t)(n0 + lane);
                // the kW gate lanes' rotation pairs (a0, a1 in one 32-bit word),
                // loaded together and then broadcast, not one dependent load
                // per iteration
                uint32_t my_a01 = 0;
                {
                    const int l = group * kGroup + d + kDrainWarps * lane;
                    if (lane < kW && l < lanes)
                        my_a01 = *reinterpret_cast<const uint32_t*>(abar + (size_t)l * 640 + 2 * pair);
                }
#pragma unroll 1
                for (int i = 0; i < kW; i++) {
                    const int gl = d + kDrainWarps * i, l = group * kGroup + gl;
                    const uint32_t v = red[(size_t)gl * kRowsCoef + lane];
                    red[(size_t)gl * kRowsCoef + lane] = 0u;
                    const uint32_t a01 = __shfl_sync(0xffffffffu, my_a01, i);
                    if (l < lanes) {
                        const uint32_t a0 = a01 & 0xFFFFu, a1 = a01 >> 16;
                        const uint32_t e = key == 0 ? (a0 + a1) & (2 * kN - 1) : key == 1 ? a0 : a1;
                        const uint32_t pos = (n + e) & (2 * kN - 1);
                        uint32_t* out = acc + (size_t)l * kTrlwe + j_out * kN;
                        atomicAdd(&out[pos & (kN - 1)], pos < (uint32_t)kN ? v : 0u - v);
                        atomicAdd(&out[n], 0u - v);
                    }
                }
            } else {
#pragma unroll
                for (int i = 0; i < kW; i++) {
                    const int gl = d + kDrainWarps * i, l = group * kGroup + gl;
                    const uint32_t v = red[(size_t)gl * kRowsCoef + lane];
                    red[(size_t)gl * kRowsCoef + lane] = 0u;
                    if (l < lanes) atomicAdd(&acc[(size_t)l * kTrlwe + j_out * kN + n0 + lane], v);
                }
            }
            __threadfence_block();
            __syncwarp();
            if (lane == 0) mbar_arrive(red_clear);
            if (!__all_sync(0xffffffffu, mbar_wait(red_clear, (uint32_t)it & 1))) {
                ok = false;
                break;
            }
        }
        if (!ok) s_fail = 1;
    }

    __syncthreads();
    if (s_fail && tid == 0) {
        atomicOr(err, 1);
        // wait (bounded) for copies and MMA batches that may be in flight (the
        // chunk barriers, which count both CTAs' copies, live in the even CTA)
        if (rank == 0)
            for (int s = 0; s < kPairStages; s++) mbar_wait(&full[s], 0), mbar_wait(&full[s], 1);
        mbar_wait(acc_full, 0), mbar_wait(acc_full, 1);
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();  // the pair's MMAs and copies are done with both CTAs' TMEM and smem
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols));
}

// SampleExtract (index 0) and accumulator copy-out
__global__ void k_i8_extract(const uint32_t* __restrict__ acc, int lanes,
                             uint32_t* __restrict__ acc_out, uint32_t* __restrict__ lane_out)
{
    const int l = blockIdx.x;
    if (l >= lanes) return;
    const uint32_t* a = acc + (size_t)l * kTrlwe;
    if (acc_out)
        for (int i = threadIdx.x; i < kTrlwe; i += blockDim.x) acc_out[(size_t)l * kTrlwe + i] = a[i];
    if (lane_out)
        for (int i = threadIdx.x; i <= kN; i += blockDim.x)
            lane_out[(size_t)l * kTlwe1 + i] = i == kN ? a[kN] : (i == 0 ? a[0] : 0u - a[kN - i]);
}

cudaError_t ensure_ws(Int8Workspace& w, int lanes, cudaStream_t st)
{
    if ((size_t)lanes <= w.cap) return cudaSuccess;
    int8_workspace_free(w);
    const int groups = (lanes + kGroup - 1) / kGroup;
    cudaError_t e;
    if ((e = cudaMalloc(&w.acc, (size_t)lanes * kTrlwe * 4)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.abar, (size_t)lanes * 640 * 2)) != cudaSuccess) return e;
    if ((e = cudaMalloc((void**)&w.digits, (size_t)groups * kChunks * kTileBytes)) != cudaSuccess) return e;
    // zeroed on the stream of the launches that use it: the engine's streams
    // are non-blocking, so a memset on the legacy stream would not be ordered
    // before (and could land after) the first decompose's stores
    e = cudaMemsetAsync(w.digits, 0, (size_t)groups * kChunks * kTileBytes, st);
    if (e != cudaSuccess) return e;
    w.cap = (size_t)lanes;
    return cudaSuccess;
}

cudaError_t set_gemm_attr()
{
    static DeviceAttrFlags attr_plain, attr_kb, attr_pair_plain, attr_pair_kb;
    cudaError_t e = set_smem_attr_once(attr_plain, k_i8_gemm_p<false>, kSmemGemmP);
    if (e == cudaSuccess) e = set_smem_attr_once(attr_kb, k_i8_gemm_p<true>, kSmemGemmP);
    if (e == cudaSuccess) e = set_smem_attr_once(attr_pair_plain, k_i8_gemm_2sm<false>, kSmemGemmPair);
    if (e == cudaSuccess) e = set_smem_attr_once(attr_pair_kb, k_i8_gemm_2sm<true>, kSmemGemmPair);
    return e;
}

// CTA pairs of the pair GEMM that can be resident at once on this device
// (SMs of a GPC pair up; an odd one is left out), cached per device
int max_pairs(int dev, int sms)
{
    static std::atomic<int> cache[64];
    const int c = cache[dev & 63].load();
    if (c > 0) return c;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * (sms / 2));
    cfg.blockDim = dim3(kGemmPThreads);
    cfg.dynamicSmemBytes = kSmemGemmPair;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_i8_gemm_2sm<true>, &cfg) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        n = sms / 2;
    }
    if (n > sms / 2) n = sms / 2;
    cache[dev & 63].store(n);
    return n;
}

// Tensor map of a workspace's digit tiles for the odd CTA's copies: rows of
// 128 bytes ([group][chunk][256 lanes] rows, already in the MMA's swizzled
// order, copied as they are), boxes of 128 rows.  cuTensorMapEncodeTiled comes
// from the driver through the runtime's entry-point query.
cudaError_t digits_tensor_map(const Int8Workspace& w, int groups, CUtensorMap* map)
{
    typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                    const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                    const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                    CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static std::atomic<EncodeTiled> encode{nullptr};
    EncodeTiled fn = encode.load();
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !f) return cudaErrorNotSupported;
        fn = reinterpret_cast<EncodeTiled>(f);
        encode.store(fn);
    }
    const cuuint64_t dims[2] = {(cuuint64_t)kChunkK, (cuuint64_t)groups * kChunks * kGroup};
    const cuuint64_t strides[1] = {(cuuint64_t)kChunkK};
    const cuuint32_t box[2] = {(cuuint32_t)kChunkK, 128u};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, w.digits, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

bool use_pair_gemm()
{
    const char* e = getenv("CUFHE_I8_PAIR");
    return !(e && e[0] == '0');
}

}  // namespace

cudaError_t int8_key_build(Int8Key& k, const uint32_t* bk_dev, bool kb, cudaStream_t st)
{
    int8_key_free(k);
    const int ntrgsw = kb ? 3 * (kN0 / 2) : kN0;
    k.bytes = (size_t)ntrgsw * kVBytesStep;
    cudaError_t e = cudaMalloc(&k.limbs, k.bytes);
    if (e != cudaSuccess) return e;
    const size_t units = k.bytes / 4;
    k_i8_key<<<(unsigned)((units + 255) / 256), 256, 0, st>>>(bk_dev, ntrgsw, (int8_t*)k.limbs);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k.kb = kb;
    k.ready = true;
    return cudaSuccess;
}

void int8_key_free(Int8Key& k)
{
    if (k.limbs) cudaFree(k.limbs);
    k = Int8Key();
}

void int8_workspace_free(Int8Workspace& w)
{
    cudaFree(w.acc);
    cudaFree(w.abar);
    cudaFree(w.digits);
    w = Int8Workspace();
}

cudaError_t int8_reserve(Int8Workspace& w, int lanes, cudaStream_t st)
{
    const cudaError_t e = ensure_ws(w, lanes, st);
    return e != cudaSuccess ? e : set_gemm_attr();
}

cudaError_t launch_br_int8(const Int8Key& k, Int8Workspace& w, const uint32_t* lane_in, int lanes,
                           uint32_t mu, int steps, uint32_t* acc_out, uint32_t* lane_out,
                           int* err, cudaStream_t st, int* launches)
{
    *launches = 0;
    if (lanes <= 0) return cudaSuccess;
    cudaError_t e = int8_reserve(w, lanes, st);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // plain key: one GEMM step per CMUX step (636); KeyBundle key: one per
    // pair (318), over the pair's three keys
    const int total = k.kb ? kN0 / 2 : kN0;
    const int nsteps = (steps < 0 || steps > total) ? total : steps;
    const int combos = k.kb ? 6 : 2;
    const size_t key_step = (size_t)(k.kb ? 3 : 1) * kVBytesStep;
    const int groups = (lanes + kGroup - 1) / kGroup;
    k_i8_init<<<lanes, 256, 0, st>>>(lane_in, lanes, mu, w.abar, w.acc);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int n = 1;
    // tiles per combo; the tiles of the last, partial round are split along
    // K so that the round's units fit one per CTA (split = 1, 2, 4 or 8).
    // Pair form: one unit per CTA pair (its two CTAs serve the two output
    // polynomials of one key), so the units per combo are the pairs per key.
    const bool pair_form = use_pair_gemm();
    CUtensorMap tmap;
    if (pair_form && (e = digits_tensor_map(w, groups, &tmap)) != cudaSuccess) return e;
    const int tiles_j = groups * (kN / kRowsCoef);
    const int keys = k.kb ? 3 : 1;
    const int ncj = pair_form ? max_pairs(dev, sms) / keys : sms / combos;
    const int rem = tiles_j % ncj;
    int split = 1;
    while (rem && split < 8 && rem * split * 2 <= ncj) split *= 2;
    const int units = tiles_j < ncj ? tiles_j * split : ncj;
    for (int i = 0; i < nsteps; i++) {
        // both kernels are programmatic dependents of the one before: each
        // starts (TMEM, barriers, key window) while the previous one drains
        cudaLaunchAttribute pdl[1];
        pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        pdl[0].val.programmaticStreamSerializationAllowed = 1;
        {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(lanes);
            cfg.blockDim = dim3(256);
            cfg.stream = st;
            cfg.attrs = pdl;
            cfg.numAttrs = 1;
            e = k.kb ? cudaLaunchKernelEx(&cfg, k_i8_decompose<true>, w.acc, (const uint16_t*)w.abar,
                                          lanes, i, (uint8_t*)w.digits)
                     : cudaLaunchKernelEx(&cfg, k_i8_decompose<false>, w.acc,
                                          (const uint16_t*)w.abar, lanes, i, (uint8_t*)w.digits);
            if (e != cudaSuccess) return e;
        }
        const int8_t* vk = (const int8_t*)k.limbs + (size_t)i * key_step;
        {
            cudaLaunchConfig_t cfg = {};
            // both forms: combos x units CTAs (pair form: keys x units pairs)
            cfg.gridDim = dim3(combos * units);
            cfg.blockDim = dim3(kGemmPThreads);
            cfg.dynamicSmemBytes = pair_form ? kSmemGemmPair : kSmemGemmP;
            cfg.stream = st;
            cfg.attrs = pdl;
            cfg.numAttrs = 1;
            const uint8_t* dg = (const uint8_t*)w.digits;
            const uint16_t* ab = (const uint16_t*)w.abar;
            if (pair_form)
                e = k.kb ? cudaLaunchKernelEx(&cfg, k_i8_gemm_2sm<true>, tmap, vk, dg, w.acc, lanes,
                                              tiles_j, split, ab, i, err)
                         : cudaLaunchKernelEx(&cfg, k_i8_gemm_2sm<false>, tmap, vk, dg, w.acc,
                                              lanes, tiles_j, split, ab, i, err);
            else
                e = k.kb ? cudaLaunchKernelEx(&cfg, k_i8_gemm_p<true>, vk, dg, w.acc, lanes,
                                              tiles_j, split, ab, i, err)
                         : cudaLaunchKernelEx(&cfg, k_i8_gemm_p<false>, vk, dg, w.acc, lanes,
                                              tiles_j, split, ab, i, err);
            if (e != cudaSuccess) return e;
        }
        n += 2;
    }
    k_i8_extract<<<lanes, 256, 0, st>>>(w.acc, lanes, acc_out, lane_out);
    n++;
    *launches = n;
    return cudaGetLastError();
}

}  // namespace cufhe
