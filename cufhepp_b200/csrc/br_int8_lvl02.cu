// Exact INT8 tensor-core blind rotation lvl0 -> lvl2 (tcgen05, sm_100a),
// plain CMUX form and KeyBundle form (one step per pair, three key GEMMs whose
// products enter as (X^e - 1) P, plus the gadget recomposition of the digits,
// as at lvl1 in br_int8.cu): the lvl02param instantiation of __BlindRotate__
// (include/gatebootstrapping_gpu.cuh:801-884) that the *_lvl02 gates run
// (src/cufhe_gates_gpu.cu:826-979), with N = 2048, l = 4, Bgbit = 10,
// Torus64.
//
// Step i is acc += ExtProd(BK_i, X^abar acc - acc), i.e. for every lane and
// output polynomial j_out
//   out[j_out][n] = sum_{r, m} dec_r[m] * sign(n, m) * BK_i[r][j_out][(n - m) mod N]
// with r = j*4 + d and signed 10-bit gadget digits dec_r in [-512, 512)
// (include/gatebootstrapping_gpu.cuh:20-29, 110-146 at lvl2param).
//
// Exactness.  Key words are split into eight balanced signed byte limbs
// (v = sum_c s_c 2^(8c) mod 2^64) and every digit into two signed limbs
// (dec = 32 d1 + d0, d0 in [-16, 16), d1 in [-16, 16]).  A K = 16384 sum of
// limb products is bounded by 16384 * 128 * 16 = 2^25 in INT32, and
// sum_{c,e} acc_{c,e} 2^(8c + 5e) mod 2^64 is the exact Torus64 product: the
// rotation is bit-identical to the schoolbook oracle.
//
// Layout.
//  * key   : for step i, output poly j, row r, limb c the 2N-byte sequence
//            V[t] = limb_c(BK[N-1-t]) (t < N), limb_c(-BK[2N-1-t]) (t >= N),
//            so Toeplitz row n over columns [m0, m0+128) is the contiguous
//            window V[N-1-n+m0 ..): [636][2][8][8][4096] int8 = 333 MB.
//  * digits: per group of 128 lanes and K chunk of 128, a 32 KB tile in the
//            canonical K-major 128B-swizzled layout whose 256 rows are
//            (digit limb e, lane): row e*128 + lane.
//  * acc   : [lanes][2][2048] Torus64.
//
// k_i82_gemm (one launch per step, one CTA per SM): tile = (128-lane group,
// 32 coefficients of one j_out, limb group lg = limbs 4lg..4lg+3), M = 128
// rows (limb, coefficient), N = 256 columns (digit limb, lane), K = 16384.
// CTA b serves output polynomial b & 1; both limb groups of a coefficient
// block run back to back on the same CTA, so every accumulator word has a
// single writer.  The structure is that of the lvl1 kernel (br_int8.cu):
// generators write Toeplitz A chunks into TMEM, one thread issues
// tcgen05.mma.kind::i8 M128 N256 K32, one thread streams digit chunks
// through a 5-stage ring with one full and one empty barrier per chunk,
// sixteen drain warps fold the limbs into the global accumulator.  The key
// windows of a tile (8.1 KB per digit row and limb group) stream through a
// two-slot ring of their own from a second producer.  Every wait is bounded
// and reports through an error flag.
#include <stdio.h>

#include "br_int8.h"
#include "engine.h"
#include "tc_util.cuh"

namespace cufhe {

namespace {

constexpr int kN2 = CUFHE_LVL2_N;              // 2048
constexpr int kTlwe2 = CUFHE_TLWE2_WORDS;      // 2049
constexpr int kTrlwe2 = CUFHE_TRLWE2_WORDS;    // 4096
constexpr int kGroup2 = 128;                   // lanes per digit group
constexpr int kChunkK = 128;                   // K bytes per chunk (one swizzle row)
constexpr int kChunks2 = 8 * kN2 / kChunkK;    // 128 chunks per tile
constexpr int kChunksPerRow = kN2 / kChunkK;   // 16 chunks per digit row r
constexpr int kTileBytes = 2 * kGroup2 * kChunkK;  // 32 KB (2 digit limbs x 128 lanes)
constexpr int kRowsCoef = 32;                  // coefficients per tile (x 4 limbs = 128 rows)
constexpr int kNBlocks = kN2 / kRowsCoef;      // 64 coefficient blocks per output poly
constexpr size_t kVRow = 2 * kN2;              // bytes per (step, j, r, limb) sequence
constexpr size_t kVStep = 2 * 8 * 8 * kVRow;   // 512 KB of key table per step
constexpr int kVWin = 2080;                    // staged window per (tile, r, limb)
constexpr int kVStage = 4 * kVWin;             // one digit row, four limbs
constexpr int kAbarStride = 640;
constexpr uint64_t kDecOffset2 = (512ull << 54) + (512ull << 44) + (512ull << 34) +
                                 (512ull << 24) + (1ull << 23);

constexpr int kPStages = 5;
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kAccCol = 0;   // accumulator columns [0, 256)
constexpr uint32_t kACol = 256;   // A slots: 32 columns each from column 256
constexpr uint32_t kIdesc = idesc_i8(128, 256);
constexpr size_t kSmemB = (size_t)kPStages * kTileBytes;     // 160 KB
constexpr size_t kSmemV = 2 * (size_t)kVStage;                // 16.3 KB
constexpr size_t kRedWords = (size_t)kGroup2 * kRowsCoef;     // 4096 (u64)
constexpr size_t kSmemRed = kRedWords * 8;                    // 32 KB
constexpr size_t kSmemGemm = 1024 + kSmemB + kSmemV + kSmemRed + 512;
constexpr int kDrainWarps = 16;
constexpr int kVWarp = 10 + kDrainWarps;                      // key-window producer
constexpr int kGemmThreads = 32 * (kVWarp + 1);               // 864

// balanced signed byte limb c of a Torus64 word: v = sum_c s_c 2^(8c) mod 2^64
__device__ __forceinline__ int8_t limb64(uint64_t v, int c)
{
    int8_t s = 0;
    for (int i = 0; i <= c; i++) {
        s = (int8_t)((int)((v + 128u) & 255u) - 128);
        v = (v - (uint64_t)(int64_t)s) >> 8;
    }
    return s;
}

// key table: out[i][j][r][c][t], t < 2N (4 bytes per thread), i over the
// key's ntrgsw TRGSWs (636 plain, 318 x 3 KeyBundle)
__global__ void k_i82_key(const uint64_t* __restrict__ bk, int ntrgsw, int8_t* __restrict__ out)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // 4-byte unit
    const size_t total = (size_t)ntrgsw * kVStep / 4;
    if (q >= total) return;
    const size_t byte = q * 4;
    const int t0 = (int)(byte % kVRow);
    size_t rest = byte / kVRow;
    const int c = (int)(rest % 8);
    rest /= 8;
    const int r = (int)(rest % 8);
    rest /= 8;
    const int j = (int)(rest % 2);
    const size_t i = rest / 2;
    const uint64_t* poly = bk + ((i * 8 + r) * 2 + j) * kN2;  // TFHEpp TRGSW[i][r][j][N]
    uint32_t packed = 0;
    for (int e = 0; e < 4; e++) {
        const int t = t0 + e;
        const uint64_t x = t < kN2 ? poly[kN2 - 1 - t] : 0ull - poly[2 * kN2 - 1 - t];
        packed |= (uint32_t)(uint8_t)limb64(x, c) << (8 * e);
    }
    reinterpret_cast<uint32_t*>(out)[q] = packed;
}

// modulus switch + test vector at lvl2 (bar = 2N - (b >> 20) unrounded,
// abar = (a + 2^19) >> 20 rounded)
__global__ void k_i82_init(const uint32_t* __restrict__ lane_in, int lanes, uint64_t mu,
                           uint16_t* __restrict__ abar, uint64_t* __restrict__ acc)
{
    const int l = blockIdx.x;
    if (l >= lanes) return;
    const uint32_t* x = lane_in + (size_t)l * kTlwe0;
    for (int i = threadIdx.x; i < kN0; i += blockDim.x)
        abar[(size_t)l * kAbarStride + i] = (uint16_t)((x[i] + (1u << 19)) >> 20);
    const uint32_t bar = 2u * kN2 - (x[kN0] >> 20);
    uint64_t* a = acc + (size_t)l * kTrlwe2;
    for (int i = threadIdx.x; i < kN2; i += blockDim.x) {
        a[i] = 0;
        a[kN2 + i] = bar == 2u * kN2
                         ? mu
                         : ((((uint32_t)i < (bar & (kN2 - 1))) ^ (bar >> 11)) ? 0ull - mu : mu);
    }
}

// Digit limbs of the step's external-product input, written as swizzled
// tiles tiles[group][chunk][32 KB]; one CTA (256 threads) per lane, 4
// coefficients per thread and pass.
//  * plain CMUX step `step`: digits of X^abar acc - acc (acc is only read);
//  * KeyBundle pair (KB): digits of acc itself, and acc is overwritten in
//    place with their gadget recomposition sum_d dec_d 2^(64 - 10 (d + 1)) =
//    (acc + 2^23) & ~(2^24 - 1), the H term to which the pair's GEMM adds the
//    rotated products.  Each thread reads and rewrites only its own words.
template <bool KB>
__global__ void __launch_bounds__(256) k_i82_decompose(uint64_t* __restrict__ acc,
                                                       const uint16_t* __restrict__ abar,
                                                       int lanes, int step,
                                                       uint8_t* __restrict__ tiles)
{
    // launched as a programmatic dependent of the previous step's GEMM: wait
    // for its accumulator updates before reading the accumulator
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int l = blockIdx.x;
    if (l >= lanes) return;
    const uint32_t ab = KB ? 0u : abar[(size_t)l * kAbarStride + step];
    const uint32_t abm = ab & (kN2 - 1), abn = ab >> 11;
    const uint32_t row = (uint32_t)(l % kGroup2);
    uint8_t* gtile = tiles + (size_t)(l / kGroup2) * kChunks2 * kTileBytes;
#pragma unroll 1
    for (int j = 0; j < 2; j++) {
        uint64_t* a = acc + (size_t)l * kTrlwe2 + j * kN2;
#pragma unroll 1
        for (int pass = 0; pass < 2; pass++) {
            const int m = (threadIdx.x + 256 * pass) * 4;
            uint32_t p0[4] = {0, 0, 0, 0}, p1[4] = {0, 0, 0, 0};
#pragma unroll
            for (int e4 = 0; e4 < 4; e4++) {
                const uint32_t n = (uint32_t)(m + e4);
                uint64_t t;
                if (KB) {
                    const uint64_t x = a[n];
                    a[n] = (x + (1ull << 23)) & ~((1ull << 24) - 1);
                    t = x + kDecOffset2;
                } else {
                    uint64_t rv = a[(n - ab) & (kN2 - 1)];
                    rv = ((n < abm) ^ abn) ? 0ull - rv : rv;
                    t = rv - a[n] + kDecOffset2;
                }
#pragma unroll
                for (int d = 0; d < 4; d++) {
                    const int dig = (int)((t >> (54 - 10 * d)) & 1023u) - 512;
                    const int d0 = ((dig + 16) & 31) - 16;
                    const int d1 = (dig - d0) >> 5;
                    p0[d] |= (uint32_t)(uint8_t)d0 << (8 * e4);
                    p1[d] |= (uint32_t)(uint8_t)d1 << (8 * e4);
                }
            }
#pragma unroll
            for (int d = 0; d < 4; d++) {
                const uint32_t K = (uint32_t)((j * 4 + d) * kN2 + m);
                uint8_t* t = gtile + (size_t)(K / kChunkK) * kTileBytes;
                *reinterpret_cast<uint32_t*>(t + swz_offset(row, K % kChunkK)) = p0[d];
                *reinterpret_cast<uint32_t*>(t + swz_offset(kGroup2 + row, K % kChunkK)) = p1[d];
            }
        }
    }
}

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

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(addr)
        : "memory");
}

// Roles: warps 0-7 generators (warpgroup wg writes the chunks of parity wg),
// warp 8 MMA issue, warp 9 digit-chunk producer, warps 10-25 drainers, warp 26
// key-window producer.  KeyBundle form (KB): CTA b serves combo b mod 6 =
// key * 2 + output polynomial of the pair's three keys, and the drain adds
// each product word P[n] at n + e (negacyclic) and subtracts it at n
// (e = a0 + a1, a0, a1 for bk0, bk1, bk2) with 64-bit atomic adds, since
// three keys add into every accumulator word.
template <bool KB>
__global__ void __launch_bounds__(kGemmThreads, 1) k_i82_gemm(const int8_t* __restrict__ vkey,
                                                              const uint8_t* __restrict__ tiles,
                                                              uint64_t* __restrict__ acc,
                                                              int lanes, int blocks_j,
                                                              const uint16_t* __restrict__ abar,
                                                              int pair, int* __restrict__ err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t raw_addr = smem_u32(smem_raw);
    unsigned char* smem = smem_raw + ((1024u - (raw_addr & 1023u)) & 1023u);
    unsigned char* bst = smem;
    int8_t* vbuf = reinterpret_cast<int8_t*>(smem + kSmemB);
    uint64_t* red = reinterpret_cast<uint64_t*>(smem + kSmemB + kSmemV);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kSmemB + kSmemV + kSmemRed);
    uint64_t* full = bars;                    // [kPStages]
    uint64_t* empty = full + kPStages;        // [kPStages]
    uint64_t* vfull = empty + kPStages;       // [2]
    uint64_t* vempty = vfull + 2;             // [2]
    uint64_t* acc_full = vempty + 2;
    uint64_t* acc_empty = acc_full + 1;
    uint64_t* red_full = acc_empty + 1;
    uint64_t* red_clear = red_full + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(red_clear + 1);
    __shared__ volatile int s_fail;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int kCombos = KB ? 6 : 2;
    const int combo = (int)(blockIdx.x % kCombos), j_out = combo & 1;
    const int cb = (int)(blockIdx.x / kCombos), ncj = (int)(gridDim.x / kCombos);
    // blocks = (group, coefficient block) pairs of this output poly; each is
    // two tiles (limb groups 0 and 1) in a row
    const int nblk = cb < blocks_j ? (blocks_j - 1 - cb) / ncj + 1 : 0;
    const int T = 2 * nblk;

    for (size_t i = tid; i < kRedWords; i += blockDim.x) red[i] = 0ull;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        s_fail = 0;
        for (int s = 0; s < kPStages; s++) {
            mbar_init(&full[s], 128 + 1);
            mbar_init(&empty[s], 1);
        }
        for (int s = 0; s < 2; s++) {
            mbar_init(&vfull[s], 1);
            mbar_init(&vempty[s], 8);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, kDrainWarps);
        mbar_init(red_full, kDrainWarps);
        mbar_init(red_clear, kDrainWarps);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 9) {
        // ---- digit-chunk producer
        if (lane == 0) {
            // the digit tiles are the previous kernel's output (programmatic
            // dependent launch)
            asm volatile("griddepcontrol.wait;" ::: "memory");
            for (int it = 0; it < T && !s_fail; it++) {
                const int group = (cb + (it >> 1) * ncj) / kNBlocks;
                const uint8_t* gt = tiles + (size_t)group * kChunks2 * kTileBytes;
                for (int kc = 0; kc < kChunks2; kc++) {
                    const int gc = it * kChunks2 + kc, s = gc % kPStages;
                    if (s_fail) break;
                    if (gc >= kPStages &&
                        !mbar_wait(&empty[s], (uint32_t)((gc / kPStages) - 1) & 1)) {
                        s_fail = 1;
                        break;
                    }
                    mbar_expect_tx(&full[s], kTileBytes);
                    bulk_g2s(bst + s * kTileBytes, gt + (size_t)kc * kTileBytes, kTileBytes, &full[s]);
                }
            }
        }
    } else if (warp == kVWarp) {
        // ---- key-window producer: per tile and digit row, the windows of the
        // tile's four limbs (bytes [2016 - n0, 4096 - n0) of each sequence)
        if (lane == 0) {
            for (int it = 0; it < T && !s_fail; it++) {
                const int blk = cb + (it >> 1) * ncj, lg = it & 1;
                const int n0 = (blk % kNBlocks) * kRowsCoef;
                for (int r = 0; r < 8; r++) {
                    const int gv = it * 8 + r, vs = gv & 1;
                    if (s_fail) break;
                    if (gv >= 2 && !mbar_wait(&vempty[vs], (uint32_t)((gv >> 1) - 1) & 1)) {
                        s_fail = 1;
                        break;
                    }
                    mbar_expect_tx(&vfull[vs], (uint32_t)kVStage);
#pragma unroll 1
                    for (int q = 0; q < 4; q++) {
                        const int c = 4 * lg + q;
                        const int8_t* src = vkey + ((size_t)(combo * 8 + r) * 8 + c) * kVRow +
                                            (2016 - n0);
                        bulk_g2s(vbuf + vs * kVStage + q * kVWin, src, (uint32_t)kVWin, &vfull[vs]);
                    }
                }
            }
        }
    } else if (warp == 8) {
        // ---- MMA issue
        if (lane == 0) {
            int gc = 0;
            for (int it = 0; it < T && !s_fail; it++) {
                if (it >= 1 && !mbar_wait(acc_empty, (uint32_t)(it - 1) & 1)) {
                    s_fail = 1;
                    break;
                }
                tc_fence_after();
                for (int kc = 0; kc < kChunks2; kc++, gc++) {
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
                                  desc_kmajor_sw128(bbase + 32 * k), kIdesc, (kc | k) != 0);
                    tc_commit(&empty[s]);
                }
                if (s_fail) break;
                tc_commit(acc_full);
            }
        }
    } else if (warp < 8) {
        // ---- generators: row (limb 4 lg + q, coefficient n0 + lane) of the
        // tile's Toeplitz block, warpgroup wg writes the chunks of parity wg
        const int wg = warp >> 2, q = warp & 3;
        const uint32_t lane_base = (uint32_t)(32 * q) << 16;
        bool ok = true;
        for (int it = 0; it < T && ok; it++) {
            for (int kc = wg; kc < kChunks2; kc += 2) {
                const int gc = it * kChunks2 + kc, s = gc % kPStages;
                const int r = kc / kChunksPerRow, m0 = (kc % kChunksPerRow) * kChunkK;
                const int gv = it * 8 + r, vs = gv & 1;
                if (__any_sync(0xffffffffu, s_fail != 0)) {
                    ok = false;
                    break;
                }
                if ((kc % kChunksPerRow) == wg &&
                    !__all_sync(0xffffffffu, mbar_wait(&vfull[vs], (uint32_t)(gv >> 1) & 1))) {
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
                const uint32_t* vw =
                    reinterpret_cast<const uint32_t*>(vbuf + vs * kVStage + q * kVWin);
                const int loc = 31 - lane + m0;  // window offset of V[N-1-n+m0]
                const int w0 = loc >> 2, sh = (loc & 3) * 8;
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
                if ((kc % kChunksPerRow) == kChunksPerRow - 2 + wg) {
                    // this warp's last chunk of digit row r: release the window slot
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&vempty[vs]);
                }
            }
        }
        if (!ok) s_fail = 1;
    } else {
        // ---- drainers: warp d reads TMEM lane quadrant warp % 4 (the hardware
        // ties a warp to quadrant warp % 4): lanes [32 p, 32 p + 32) of both
        // digit limbs (columns 32 p + i and 128 + 32 p + i)
        const int d = warp - 10, q = warp & 3, p = d >> 2;
        const uint32_t lane_base = (uint32_t)(32 * q) << 16;
        asm volatile("griddepcontrol.wait;" ::: "memory");
        bool ok = true;
        for (int it = 0; it < T && ok; it++) {
            const int blk = cb + (it >> 1) * ncj, lg = it & 1;
            const int group = blk / kNBlocks;
            const int n0 = (blk % kNBlocks) * kRowsCoef;
            const int shift = 8 * (4 * lg + q);
            if (__any_sync(0xffffffffu, s_fail != 0) ||
                !__all_sync(0xffffffffu, mbar_wait(acc_full, (uint32_t)it & 1))) {
                ok = false;
                break;
            }
            tc_fence_after();
#pragma unroll 1
            for (int hh = 0; hh < 2; hh++) {
                uint32_t v0[16], v1[16];
                tmem_ld16(tmem + lane_base + kAccCol + 32 * p + 16 * hh, v0);
                tmem_ld16(tmem + lane_base + kAccCol + kGroup2 + 32 * p + 16 * hh, v1);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const uint64_t v = ((uint64_t)(int64_t)(int32_t)v0[i] +
                                        ((uint64_t)(int64_t)(int32_t)v1[i] << 5))
                                       << shift;
                    atomicAdd(reinterpret_cast<unsigned long long*>(
                                  &red[(size_t)(32 * p + 16 * hh + i) * kRowsCoef + lane]),
                              (unsigned long long)v);
                }
            }
            tc_fence_before();
            __threadfence_block();  // this warp's shared-buffer adds before the hand-off
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(acc_empty);
                mbar_arrive(red_full);
            }
            if (!__all_sync(0xffffffffu, mbar_wait(red_full, (uint32_t)it & 1))) {
                ok = false;
                break;
            }
            constexpr int kW = kGroup2 / kDrainWarps;  // 8 lanes per warp
            if (KB) {
                const int key = combo >> 1;
                const uint32_t n = (uint32_t)(n0 + lane);
                // the kW gate lanes' rotation pairs, loaded together
                uint32_t my_a01 = 0;
                {
                    const int l = group * kGroup2 + d + kDrainWarps * lane;
                    if (lane < kW && l < lanes)
                        my_a01 = *reinterpret_cast<const uint32_t*>(abar + (size_t)l * kAbarStride +
                                                                    2 * pair);
                }
#pragma unroll 1
                for (int i = 0; i < kW; i++) {
                    const int gl = d + kDrainWarps * i, l = group * kGroup2 + gl;
                    const uint64_t v = red[(size_t)gl * kRowsCoef + lane];
                    red[(size_t)gl * kRowsCoef + lane] = 0ull;
                    const uint32_t a01 = __shfl_sync(0xffffffffu, my_a01, i);
                    if (l < lanes) {
                        const uint32_t a0 = a01 & 0xFFFFu, a1 = a01 >> 16;
                        const uint32_t e = key == 0 ? (a0 + a1) & (2 * kN2 - 1) : key == 1 ? a0 : a1;
                        const uint32_t pos = (n + e) & (2 * kN2 - 1);
                        unsigned long long* out = reinterpret_cast<unsigned long long*>(
                            acc + ((size_t)l * 2 + j_out) * kN2);
                        atomicAdd(&out[pos & (kN2 - 1)],
                                  (unsigned long long)(pos < (uint32_t)kN2 ? v : 0ull - v));
                        atomicAdd(&out[n], (unsigned long long)(0ull - v));
                    }
                }
            } else {
                // all loads in flight before the stores (one writer per word)
                uint64_t old[kW];
#pragma unroll
                for (int i = 0; i < kW; i++) {
                    const int l = group * kGroup2 + d + kDrainWarps * i;
                    old[i] = l < lanes ? acc[((size_t)l * 2 + j_out) * kN2 + n0 + lane] : 0ull;
                }
#pragma unroll
                for (int i = 0; i < kW; i++) {
                    const int gl = d + kDrainWarps * i, l = group * kGroup2 + gl;
                    const uint64_t v = red[(size_t)gl * kRowsCoef + lane];
                    red[(size_t)gl * kRowsCoef + lane] = 0ull;
                    if (l < lanes) acc[((size_t)l * 2 + j_out) * kN2 + n0 + lane] = old[i] + v;
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
        for (int s = 0; s < 2; s++) mbar_wait(&vfull[s], 0), mbar_wait(&vfull[s], 1);
        mbar_wait(acc_full, 0), mbar_wait(acc_full, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols));
}

// SampleExtract (index 0) at lvl2 and accumulator copy-out
__global__ void k_i82_extract(const uint64_t* __restrict__ acc, int lanes,
                              uint64_t* __restrict__ acc_out, uint64_t* __restrict__ lane_out)
{
    const int l = blockIdx.x;
    if (l >= lanes) return;
    const uint64_t* a = acc + (size_t)l * kTrlwe2;
    if (acc_out)
        for (int i = threadIdx.x; i < kTrlwe2; i += blockDim.x)
            acc_out[(size_t)l * kTrlwe2 + i] = a[i];
    if (lane_out)
        for (int i = threadIdx.x; i <= kN2; i += blockDim.x)
            lane_out[(size_t)l * kTlwe2 + i] =
                i == kN2 ? a[kN2] : (i == 0 ? a[0] : 0ull - a[kN2 - i]);
}

cudaError_t ensure_ws2(Int8Workspace2& w, int lanes, cudaStream_t st)
{
    if ((size_t)lanes <= w.cap) return cudaSuccess;
    int8_workspace2_free(w);
    const int groups = (lanes + kGroup2 - 1) / kGroup2;
    const size_t dbytes = (size_t)groups * kChunks2 * kTileBytes;
    cudaError_t e;
    if ((e = cudaMalloc(&w.acc, (size_t)lanes * kTrlwe2 * 8)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.abar, (size_t)lanes * kAbarStride * 2)) != cudaSuccess) return e;
    if ((e = cudaMalloc((void**)&w.digits, dbytes)) != cudaSuccess) return e;
    // zeroed in stream order (the engine's streams are non-blocking)
    if ((e = cudaMemsetAsync(w.digits, 0, dbytes, st)) != cudaSuccess) return e;
    w.cap = (size_t)lanes;
    return cudaSuccess;
}

cudaError_t set_gemm2_attr()
{
    static DeviceAttrFlags attr;
    static DeviceAttrFlags attr_kb;
    const cudaError_t e = set_smem_attr_once(attr, k_i82_gemm<false>, kSmemGemm);
    return e != cudaSuccess ? e : set_smem_attr_once(attr_kb, k_i82_gemm<true>, kSmemGemm);
}

}  // namespace

cudaError_t int8_key2_build(Int8Key& k, const uint64_t* bk2_dev, bool kb, cudaStream_t st)
{
    int8_key_free(k);
    const int ntrgsw = kb ? 3 * (kN0 / 2) : kN0;
    k.bytes = (size_t)ntrgsw * kVStep;
    cudaError_t e = cudaMalloc(&k.limbs, k.bytes);
    if (e != cudaSuccess) return e;
    const size_t units = k.bytes / 4;
    k_i82_key<<<(unsigned)((units + 255) / 256), 256, 0, st>>>(bk2_dev, ntrgsw, (int8_t*)k.limbs);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k.kb = kb;
    k.ready = true;
    return cudaSuccess;
}

void int8_workspace2_free(Int8Workspace2& w)
{
    cudaFree(w.acc);
    cudaFree(w.abar);
    cudaFree(w.digits);
    w = Int8Workspace2();
}

cudaError_t int8_reserve2(Int8Workspace2& w, int lanes, cudaStream_t st)
{
    const cudaError_t e = ensure_ws2(w, lanes, st);
    return e != cudaSuccess ? e : set_gemm2_attr();
}

cudaError_t launch_br2_int8(const Int8Key& k, Int8Workspace2& w, const uint32_t* lane_in, int lanes,
                            uint64_t mu, int steps, uint64_t* acc_out, uint64_t* lane_out,
                            int* err, cudaStream_t st, int* launches)
{
    *launches = 0;
    if (lanes <= 0) return cudaSuccess;
    cudaError_t e = int8_reserve2(w, lanes, st);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // plain key: one GEMM step per CMUX step (636); KeyBundle key: one per
    // pair (318) over the pair's three keys
    const int total = k.kb ? kN0 / 2 : kN0;
    const int nsteps = (steps < 0 || steps > total) ? total : steps;
    const int groups = (lanes + kGroup2 - 1) / kGroup2;
    // CTA b serves combo b mod combos (plain: the output polynomial; KeyBundle:
    // key * 2 + output polynomial)
    const int combos = k.kb ? 6 : 2;
    const size_t key_step = (size_t)(k.kb ? 3 : 1) * kVStep;
    const int blocks_j = groups * kNBlocks;
    const int grid = combos * (blocks_j < sms / combos ? blocks_j : sms / combos);
    k_i82_init<<<lanes, 256, 0, st>>>(lane_in, lanes, mu, w.abar, w.acc);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int n = 1;
    for (int i = 0; i < nsteps; i++) {
        // both kernels are programmatic dependents of the one before: each
        // starts (TMEM, barriers, key windows) while the previous one drains
        cudaLaunchAttribute pdl[1];
        pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        pdl[0].val.programmaticStreamSerializationAllowed = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(lanes);
        cfg.blockDim = dim3(256);
        cfg.stream = st;
        cfg.attrs = pdl;
        cfg.numAttrs = 1;
        const uint16_t* ab = (const uint16_t*)w.abar;
        e = k.kb ? cudaLaunchKernelEx(&cfg, k_i82_decompose<true>, w.acc, ab, lanes, i,
                                      (uint8_t*)w.digits)
                 : cudaLaunchKernelEx(&cfg, k_i82_decompose<false>, w.acc, ab, lanes, i,
                                      (uint8_t*)w.digits);
        if (e != cudaSuccess) return e;
        const int8_t* vk = (const int8_t*)k.limbs + (size_t)i * key_step;
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(kGemmThreads);
        cfg.dynamicSmemBytes = kSmemGemm;
        const uint8_t* dg = (const uint8_t*)w.digits;
        e = k.kb ? cudaLaunchKernelEx(&cfg, k_i82_gemm<true>, vk, dg, w.acc, lanes, blocks_j, ab,
                                      i, err)
                 : cudaLaunchKernelEx(&cfg, k_i82_gemm<false>, vk, dg, w.acc, lanes, blocks_j, ab,
                                      i, err);
        if (e != cudaSuccess) return e;
        n += 2;
    }
    k_i82_extract<<<lanes, 256, 0, st>>>(w.acc, lanes, acc_out, lane_out);
    n++;
    *launches = n;
    return cudaGetLastError();
}

}  // namespace cufhe
