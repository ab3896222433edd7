// Identity key switching lvl1 -> lvl0 on the tensor cores (integer,
// bit-exact).
//
// IdentityKeySwitchPreAdd / KeySwitchFromTLWE (include/keyswitch_gpu.cuh:
// 128-256) compute, for x = ca*A + cb*B (+off on b),
//   res[o] = [o == n0] x_b + sum_{i < 1024, j < 7} c(v_ij) . KSK[i][j][.][o]
// with digits v_ij in [-2, 1]: v = -1 adds KSK[i][j][0], v = +1 subtracts it,
// v = -2 adds KSK[i][j][1].  Written over K = (i, j, e) with e in {0, 1} this
// is an exact GEMM with a one-hot operand:
//   A[gate][k] in {-1, 0, +1}  (per gate, from the digits)
//   B[k][(o, c)] = limb_c(KSK[k][o])  (balanced signed bytes, shared by all gates)
//   res[o] = x_b[o == n0] + sum_c (A B_c)[o] << 8c   mod 2^32
// K = 14336, |sum| <= 7168 * 128, so INT32 accumulation is exact.
//
// The SIMT kernel in keyswitch.cu spends ~800 K integer instructions per key
// switch; here one 128-gate x 256-column tile is 448 tcgen05.mma.kind::i8
// (M = 128, N = 256, K = 32) with both operands streamed from pre-swizzled
// tiles by cp.async.bulk through a 4-stage shared-memory ring, INT32
// accumulators in TMEM, and the limb recombination in the epilogue.
#include "engine.h"
#include "tc_util.cuh"

namespace cufhe {

namespace {

constexpr int kT = CUFHE_LVL10_T;
constexpr int kChunkK = 128;
constexpr int kMGates = 128;                // gates per tile (M)
constexpr int kNCols = 256;                 // 64 outputs x 4 limbs per tile (N)
constexpr int kOutPerTile = kNCols / 4;     // 64
constexpr int kNTiles = (kTlwe0 + kOutPerTile - 1) / kOutPerTile;  // 10
constexpr int kATile = kMGates * kChunkK;   // 16 KB
constexpr int kBTile = kNCols * kChunkK;    // 32 KB
constexpr int kStageBytes = kATile + kBTile;
constexpr int kStages = 4;
constexpr size_t kSmem = 1024 + (size_t)kStages * kStageBytes + 256;
constexpr uint32_t kIdescIks = idesc_i8(kMGates, kNCols);
constexpr uint32_t kTmemColsIks = 256;
// MT unit tiles per CTA share every key chunk (MT accumulators of 256 TMEM
// columns): a stage holds MT A tiles and one B tile.  MT = 2 halves the key
// bytes streamed per unit, for keys far larger than L2 (private key
// switching: 2.5 GB per function).
template <int MT>
constexpr int iks_stages() { return MT == 1 ? kStages : 3; }
template <int MT>
constexpr size_t iks_smem() { return 1024 + (size_t)iks_stages<MT>() * (MT * kATile + kBTile) + 256; }

// K = (i, j, e) of an input with NIN mask coefficients: NIN * 7 * 2
template <int NIN>
constexpr int iks_chunks() { return NIN * kT * 2 / kChunkK; }  // 112 (lvl1), 224 (lvl2)
constexpr int kK = kN * kT * 2;             // 14336
constexpr int kChunks = iks_chunks<kN>();

__host__ __device__ constexpr uint32_t iks_offset_tc()
{
    uint32_t off = 0;
    for (int i = 1; i <= kT; i++) off += 2u << (32 - i * CUFHE_LVL10_BASEBIT);
    return off + (1u << (32 - (1 + CUFHE_LVL10_BASEBIT * kT)));
}

// lvl20: the same decomposition of a Torus64 value (include/keyswitch_gpu.cuh
// :128-187 at lvl20param)
__host__ __device__ constexpr uint64_t iks20_offset_tc()
{
    uint64_t off = 0;
    for (int i = 1; i <= (int)CUFHE_LVL20_T; i++) off += 2ull << (64 - i * CUFHE_LVL20_BASEBIT);
    return off + (1ull << (64 - (1 + CUFHE_LVL20_BASEBIT * CUFHE_LVL20_T)));
}

// key tiles [nt][kc][32 KB]: row = o_local * 4 + c, K-major, 128B-swizzled.
// Key row k (k < KTOT) has OUTW words; rows k >= KTOT and columns o >= OUTW
// are zero.
template <int CH, int NT, int OUTW, int KTOT>
__global__ void k_iks_key(const uint32_t* __restrict__ ksk, uint8_t* __restrict__ out)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = (size_t)NT * CH * kBTile / 4;
    if (q >= total) return;
    const size_t byte = q * 4;
    const int tile = (int)(byte / kBTile);
    const uint32_t w = (uint32_t)(byte % kBTile);
    const int nt = tile / CH, kc = tile % CH;
    const uint32_t row = (w / 1024) * 8 + (w % 1024) / 128;
    const uint32_t kl = ((((w % 128) / 16) ^ (row & 7)) << 4) + (w % 16);
    const int o = nt * kOutPerTile + (int)(row / 4);
    const int c = (int)(row % 4);
    uint32_t packed = 0;
    for (int e = 0; e < 4; e++) {
        const size_t k = (size_t)kc * kChunkK + kl + e;
        const int8_t v = (o < OUTW && k < (size_t)KTOT) ? limb(ksk[k * OUTW + o], c) : (int8_t)0;
        packed |= (uint32_t)(uint8_t)v << (8 * e);
    }
    reinterpret_cast<uint32_t*>(out)[q] = packed;
}

// one-hot byte pair of digit code (v = code - 2): v = -1 -> +KSK[.][0],
// v = +1 -> -KSK[.][0], v = -2 -> +KSK[.][1]
__device__ __forceinline__ uint32_t onehot_pair(uint32_t code)
{
    const uint32_t b0 = code == 1 ? 0x01u : (code == 3 ? 0xFFu : 0u);
    const uint32_t b1 = code == 0 ? 0x01u : 0u;
    return b0 | (b1 << 8);
}

// one-hot digit tiles of unit u (a lane in mode 0, a gate in mode 1):
// atiles[u / 128][kc][16 KB], row u % 128; xb[u] = b part; valid[u]
__global__ void __launch_bounds__(256) k_iks_prep(int mode, Plan plan, const uint32_t* __restrict__ in0,
                                                  const uint32_t* __restrict__ in1,
                                                  const uint32_t* __restrict__ in2,
                                                  const uint32_t* __restrict__ lane_out,
                                                  uint8_t* __restrict__ atiles,
                                                  uint32_t* __restrict__ xb, int* __restrict__ valid)
{
    const int u = blockIdx.x;
    LanePreadd p = {nullptr, nullptr, 0, 0, 0};
    int ok = 0;
    if (mode == 0) {
        p = plan_lane_preadd(plan, u, in0, in1, in2, kTlwe1);
        ok = 1;
    } else {
        const int l0 = plan_lane0(plan, u);
        if (l0 >= 0) {
            p = gate_combine(plan_op(plan, u), lane_out + (size_t)l0 * kTlwe1,
                             lane_out + (size_t)(l0 + 1) * kTlwe1);
            ok = 1;
        }
    }
    if (threadIdx.x == 0) {
        uint32_t b = 0;
        if (ok) {
            b = (uint32_t)p.ca * p.a[kN] + p.off;
            if (p.cb) b += (uint32_t)p.cb * p.b[kN];
        }
        xb[u] = b;
        valid[u] = ok;
    }
    const uint32_t row = (uint32_t)(u % kMGates);
    uint8_t* tb = atiles + (size_t)(u / kMGates) * kChunks * kATile;
    for (int q = threadIdx.x; q < kK / 16; q += blockDim.x) {
        // 16 bytes = 8 (i, j) pairs x (e = 0, e = 1)
        uint32_t wv[4] = {0, 0, 0, 0};
        int ci = -1;
        uint32_t t = 0;
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int pr = 8 * q + e, i = pr / kT, j = pr % kT;
            if (i != ci) {
                ci = i;
                uint32_t x = 0;
                if (ok) {
                    x = (uint32_t)p.ca * p.a[i];
                    if (p.cb) x += (uint32_t)p.cb * p.b[i];
                }
                t = x + iks_offset_tc();
            }
            const uint32_t code = ok ? (t >> (30 - 2 * j)) & 3u : 2u;  // v = code - 2
            wv[e >> 1] |= onehot_pair(code) << (16 * (e & 1));
        }
        const int k0 = 16 * q;
        *reinterpret_cast<uint4*>(tb + (size_t)(k0 / kChunkK) * kATile +
                                  swz_offset(row, (uint32_t)(k0 % kChunkK))) =
            make_uint4(wv[0], wv[1], wv[2], wv[3]);
    }
}

// lvl02 gates: one-hot digit tiles of gate u from its lane outputs at lvl2
// (uint64 TLWE<lvl2>), combined as binary -> lane0, Mux -> lane0 + lane1 +
// mu2, NMux -> -(lane0 + lane1) - mu2 (src/cufhe_gates_gpu.cu:826-979);
// xb[u] = the combined b rounded to Torus32 (include/keyswitch_gpu.cuh:33-50).
__global__ void __launch_bounds__(256) k_iks20_prep(Plan plan, const uint64_t* __restrict__ lane_out,
                                                    uint8_t* __restrict__ atiles,
                                                    uint32_t* __restrict__ xb, int* __restrict__ valid)
{
    constexpr int kCh = iks_chunks<CUFHE_LVL2_N>();
    constexpr int kTl2 = CUFHE_TLWE2_WORDS;
    const int u = blockIdx.x;
    const int l0 = plan_lane0(plan, u);
    const bool ok = l0 >= 0;
    const int op = plan_op(plan, u);
    const uint64_t* A = ok ? lane_out + (size_t)l0 * kTl2 : nullptr;
    const uint64_t* B = (ok && (op == kMux || op == kNMux)) ? A + kTl2 : nullptr;
    const uint64_t neg = op == kNMux ? ~0ull : 0ull;  // x -> -x when set
    if (threadIdx.x == 0) {
        uint32_t b = 0;
        if (ok) {
            uint64_t x = A[CUFHE_LVL2_N] + (B ? B[CUFHE_LVL2_N] + CUFHE_MU64 : 0ull);
            x = (x ^ neg) - neg;
            b = (uint32_t)((x + (1ull << 31)) >> 32);
        }
        xb[u] = b;
        valid[u] = ok;
    }
    const uint32_t row = (uint32_t)(u % kMGates);
    uint8_t* tb = atiles + (size_t)(u / kMGates) * kCh * kATile;
    for (int q = threadIdx.x; q < kCh * kChunkK / 16; q += blockDim.x) {
        uint32_t wv[4] = {0, 0, 0, 0};
        int ci = -1;
        uint64_t t = 0;
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int pr = 8 * q + e, i = pr / kT, j = pr % kT;
            if (i != ci) {
                ci = i;
                uint64_t x = 0;
                if (ok) {
                    x = A[i] + (B ? B[i] : 0ull);
                    x = (x ^ neg) - neg;
                }
                t = x + iks20_offset_tc();
            }
            const uint32_t code = ok ? (uint32_t)(t >> (62 - 2 * j)) & 3u : 2u;
            wv[e >> 1] |= onehot_pair(code) << (16 * (e & 1));
        }
        const int k0 = 16 * q;
        *reinterpret_cast<uint4*>(tb + (size_t)(k0 / kChunkK) * kATile +
                                  swz_offset(row, (uint32_t)(k0 % kChunkK))) =
            make_uint4(wv[0], wv[1], wv[2], wv[3]);
    }
}

// ---- private key switching TLWE<lvl2> -> TRLWE<lvl1> as a one-hot GEMM:
// K = (i, j, u) = 2049 x 10 x 15 (i: input word, j: 4-bit digit level, u:
// digit value - 1), A[unit][k] = -1 where digit j of word i of the unit is
// u + 1, B[k][(o, c)] = limb c of key row k, word o (2048 words); each
// digit selects one row, so |sum| <= 20490 x 128 fits INT32 exactly.
constexpr int kPksT = 10;
constexpr int kPksNu = 15;
constexpr int kPksK = (CUFHE_LVL2_N + 1) * kPksT * kPksNu;           // 307,350
constexpr int kPksChunks = (kPksK + kChunkK - 1) / kChunkK;          // 2402
constexpr int kPksWordsOut = 2 * CUFHE_LVL1_N;                       // 2048
constexpr int kPksNTiles = kPksWordsOut / kOutPerTile;               // 32

__global__ void __launch_bounds__(256) k_pks_prep(const uint64_t* __restrict__ tlwe, int units,
                                                  PksMap map, uint8_t* __restrict__ atiles)
{
    const int u = blockIdx.x;
    if (u >= units) return;
    const uint64_t* t = tlwe + (size_t)u * (CUFHE_LVL2_N + 1);
    const uint64_t badd = map.badd[u / map.per];
    constexpr uint64_t kOff = 1ull << (64 - (1 + 4 * kPksT));
    const uint32_t row = (uint32_t)(u % kMGates);
    uint8_t* tb = atiles + (size_t)(u / kMGates) * kPksChunks * kATile;
    for (int q = threadIdx.x; q < kPksChunks * kChunkK / 16; q += blockDim.x) {
        uint32_t wv[4] = {0, 0, 0, 0};
        int ci = -1;
        uint64_t ab = 0;
#pragma unroll
        for (int e = 0; e < 16; e++) {
            const int k = 16 * q + e;
            if (k >= kPksK) break;
            const int c = k / (kPksT * kPksNu), rem = k % (kPksT * kPksNu);
            const int j = rem / kPksNu, uu = rem % kPksNu;
            if (c != ci) {
                ci = c;
                ab = t[c] + (c == CUFHE_LVL2_N ? badd : 0ull) + kOff;
            }
            const uint32_t d = (uint32_t)(ab >> (60 - 4 * j)) & 15u;
            if (d == (uint32_t)uu + 1) wv[e >> 2] |= 0xFFu << (8 * (e & 3));
        }
        const int k0 = 16 * q;
        *reinterpret_cast<uint4*>(tb + (size_t)(k0 / kChunkK) * kATile +
                                  swz_offset(row, (uint32_t)(k0 % kChunkK))) =
            make_uint4(wv[0], wv[1], wv[2], wv[3]);
    }
}

// Output rows of the one-hot GEMM: unit u writes OUTW words at
// dst + (idx ? idx[u] : u % per) * stride_lo + (u / per) * stride_hi.
struct OutMap {
    const int32_t* idx;
    int per;
    size_t stride_lo, stride_hi;
};

// xb (optional) is added to output word OUTW - 1; valid (optional) masks units.
template <int CH, int NT, int OUTW, int MT = 1>
__global__ void __launch_bounds__(128, 1) k_iks_gemm(const uint8_t* __restrict__ atiles,
                                                     const uint8_t* __restrict__ btiles,
                                                     const uint32_t* __restrict__ xb,
                                                     const int* __restrict__ valid, int units,
                                                     uint32_t* __restrict__ dst, OutMap om,
                                                     int* __restrict__ err)
{
    constexpr int S = iks_stages<MT>();
    constexpr int SB = MT * kATile + kBTile;  // stage bytes: MT A tiles, then the B tile
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t raw_addr = smem_u32(smem_raw);
    unsigned char* smem = smem_raw + ((1024u - (raw_addr & 1023u)) & 1023u);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)S * SB);
    uint64_t* empty = full + S;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(empty + S);
    __shared__ int s_fail;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int gt = blockIdx.x / NT, nt = blockIdx.x % NT;
    // this CTA's unit tiles: gt * MT + m for m < mc
    const int gtiles = (units + kMGates - 1) / kMGates;
    const int mc = gtiles - gt * MT < MT ? gtiles - gt * MT : MT;
    const uint8_t* ga = atiles + (size_t)gt * MT * CH * kATile;
    const uint8_t* gb = btiles + (size_t)nt * CH * kBTile;
    int pend[S];  // thread 0: 1 + parity of an outstanding fill
#pragma unroll
    for (int s = 0; s < S; s++) pend[s] = 0;
    int last_commit = -1;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(kTmemColsIks * MT));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        s_fail = 0;
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (tid == 0) {
        auto fill = [&](int s, int kc) {
            unsigned char* st = smem + (size_t)s * SB;
            mbar_expect_tx(&full[s], (uint32_t)(mc * kATile + kBTile));
            for (int m = 0; m < mc; m++)
                bulk_g2s(st + m * kATile, ga + ((size_t)m * CH + kc) * kATile, kATile, &full[s]);
            bulk_g2s(st + MT * kATile, gb + (size_t)kc * kBTile, kBTile, &full[s]);
            pend[s] = 1 + ((kc / S) & 1);
        };
        for (int s = 0; s < S; s++) fill(s, s);
        for (int kc = 0; kc < CH; kc++) {
            const int s = kc % S;
            if (!mbar_wait(&full[s], (kc / S) & 1)) {
                s_fail = 1;
                break;
            }
            pend[s] = 0;
            tc_fence_after();
            const uint32_t a0 = smem_u32(smem + (size_t)s * SB);
            const uint32_t b0 = a0 + MT * kATile;
            for (int m = 0; m < mc; m++)
#pragma unroll
                for (int k = 0; k < kChunkK / 32; k++)
                    tc_mma_i8_ss(tmem + kTmemColsIks * m, desc_kmajor_sw128(a0 + m * kATile + 32 * k),
                                 desc_kmajor_sw128(b0 + 32 * k), kIdescIks, (kc | k) != 0);
            tc_commit(&empty[s]);
            last_commit = kc;
            // refill the stage of chunk kc-1 with chunk kc+S-1 once its MMAs are done
            if (kc >= 1 && kc + S - 1 < CH) {
                const int sp = (kc - 1) % S;
                if (!mbar_wait(&empty[sp], ((kc - 1) / S) & 1)) {
                    s_fail = 1;
                    break;
                }
                fill(sp, kc + S - 1);
            }
        }
        if (!s_fail && !mbar_wait(&empty[(CH - 1) % S], ((CH - 1) / S) & 1))
            s_fail = 1;
        if (s_fail) {
            atomicOr(err, 1);
            for (int s = 0; s < S; s++)
                if (pend[s]) mbar_wait(&full[s], (uint32_t)(pend[s] - 1));
            if (last_commit >= 0)
                mbar_wait(&empty[last_commit % S], (uint32_t)((last_commit / S) & 1));
        }
    }
    __syncthreads();
    tc_fence_after();
#pragma unroll 1
    for (int m = 0; m < mc && !s_fail; m++) {
        // this thread's TMEM lane = unit row of tile gt * MT + m
        const int u = (gt * MT + m) * kMGates + warp * 32 + lane;
        const bool live = u < units && (!valid || valid[u]);
        uint32_t* rowp = dst;
        if (live)
            rowp += (om.idx ? (size_t)om.idx[u] : (size_t)(u % om.per)) * om.stride_lo +
                    (size_t)(u / om.per) * om.stride_hi;
        const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
#pragma unroll 1
        for (int cc = 0; cc < kNCols / 32; cc++) {
            uint32_t v[32];
            tmem_ld32(tmem + lane_base + kTmemColsIks * m + 32 * cc, v);
            tmem_wait_ld();
            if (live) {
#pragma unroll
                for (int oo = 0; oo < 8; oo++) {
                    const int o = nt * kOutPerTile + cc * 8 + oo;
                    uint32_t r = v[4 * oo] + (v[4 * oo + 1] << 8) + (v[4 * oo + 2] << 16) +
                                 (v[4 * oo + 3] << 24);
                    if (xb && o == OUTW - 1) r += xb[u];
                    if (o < OUTW) rowp[o] = r;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemColsIks * MT));
}

}  // namespace

size_t iks_tc_key_bytes() { return (size_t)kNTiles * kChunks * kBTile; }
size_t iks20_tc_key_bytes() { return (size_t)kNTiles * iks_chunks<CUFHE_LVL2_N>() * kBTile; }

cudaError_t iks_tc_key_build(const uint32_t* ksk_dev, uint8_t* key_tiles, cudaStream_t st)
{
    const size_t units = iks_tc_key_bytes() / 4;
    k_iks_key<kChunks, kNTiles, kTlwe0, kChunks * kChunkK>
        <<<(unsigned)((units + 255) / 256), 256, 0, st>>>(ksk_dev, key_tiles);
    return cudaGetLastError();
}

cudaError_t iks20_tc_key_build(const uint32_t* ksk_dev, uint8_t* key_tiles, cudaStream_t st)
{
    const size_t units = iks20_tc_key_bytes() / 4;
    constexpr int kCh2 = iks_chunks<CUFHE_LVL2_N>();
    k_iks_key<kCh2, kNTiles, kTlwe0, kCh2 * kChunkK>
        <<<(unsigned)((units + 255) / 256), 256, 0, st>>>(ksk_dev, key_tiles);
    return cudaGetLastError();
}

static cudaError_t iks_tc_workspace(IksWorkspace& w, int units, int chunks, cudaStream_t st)
{
    if ((size_t)units <= w.cap && chunks == w.chunks) return cudaSuccess;
    iks_tc_workspace_free(w);
    const size_t tiles = (size_t)(units + kMGates - 1) / kMGates;
    cudaError_t e;
    if ((e = cudaMalloc(&w.atiles, tiles * chunks * kATile)) != cudaSuccess) return e;
    // zeroed in stream order: the engine's streams are non-blocking, so a
    // memset on the legacy stream could land after the first prep's stores
    if ((e = cudaMemsetAsync(w.atiles, 0, tiles * chunks * kATile, st)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.xb, (size_t)units * 4)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.valid, (size_t)units * 4)) != cudaSuccess) return e;
    w.cap = (size_t)units;
    w.chunks = chunks;
    return cudaSuccess;
}

cudaError_t iks_tc_reserve(IksWorkspace& w, int units, bool lvl2, cudaStream_t st)
{
    return iks_tc_workspace(w, units, lvl2 ? iks_chunks<CUFHE_LVL2_N>() : kChunks, st);
}

void iks_tc_workspace_free(IksWorkspace& w)
{
    cudaFree(w.atiles);
    cudaFree(w.xb);
    cudaFree(w.valid);
    w = IksWorkspace();
}

template <int CH, int NT, int OUTW, int MT = 1>
static cudaError_t gemm_attr()
{
    static DeviceAttrFlags attr;
    {
        const cudaError_t e = set_smem_attr_once(attr, k_iks_gemm<CH, NT, OUTW, MT>, iks_smem<MT>());
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_iks_tc(int mode, const Plan& plan, const uint32_t* in0, const uint32_t* in1,
                          const uint32_t* in2, const uint32_t* lane_out, const uint8_t* key_tiles,
                          uint32_t* dst, IksWorkspace& w, int* err, cudaStream_t st,
                          int* launches)
{
    *launches = 0;
    const int units = mode == 0 ? plan.lanes : plan.count;
    if (units <= 0) return cudaSuccess;
    cudaError_t e = iks_tc_workspace(w, units, kChunks, st);
    if (e == cudaSuccess) e = gemm_attr<kChunks, kNTiles, kTlwe0>();
    if (e != cudaSuccess) return e;
    k_iks_prep<<<units, 256, 0, st>>>(mode, plan, in0, in1, in2, lane_out, w.atiles, w.xb, w.valid);
    const int gtiles = (units + kMGates - 1) / kMGates;
    const OutMap om = {mode == 1 ? plan.out_idx : nullptr, 0x7fffffff, (size_t)kTlwe0, 0};
    k_iks_gemm<kChunks, kNTiles, kTlwe0>
        <<<gtiles * kNTiles, 128, kSmem, st>>>(w.atiles, key_tiles, w.xb, w.valid, units, dst, om, err);
    *launches = 2;
    return cudaGetLastError();
}

cudaError_t launch_iks20_tc(const Plan& plan, const uint64_t* lane_out, const uint8_t* key_tiles,
                            uint32_t* dst, IksWorkspace& w, int* err, cudaStream_t st,
                            int* launches)
{
    constexpr int kCh = iks_chunks<CUFHE_LVL2_N>();
    *launches = 0;
    const int units = plan.count;
    if (units <= 0) return cudaSuccess;
    cudaError_t e = iks_tc_workspace(w, units, kCh, st);
    if (e == cudaSuccess) e = gemm_attr<kCh, kNTiles, kTlwe0>();
    if (e != cudaSuccess) return e;
    k_iks20_prep<<<units, 256, 0, st>>>(plan, lane_out, w.atiles, w.xb, w.valid);
    const int gtiles = (units + kMGates - 1) / kMGates;
    const OutMap om = {plan.out_idx, 0x7fffffff, (size_t)kTlwe0, 0};
    k_iks_gemm<kCh, kNTiles, kTlwe0>
        <<<gtiles * kNTiles, 128, kSmem, st>>>(w.atiles, key_tiles, w.xb, w.valid, units, dst, om, err);
    *launches = 2;
    return cudaGetLastError();
}

size_t privks_tc_key_bytes() { return (size_t)kPksNTiles * kPksChunks * kBTile; }

cudaError_t privks_tc_key_build(const uint32_t* key_dev, uint8_t* key_tiles, cudaStream_t st)
{
    const size_t units = privks_tc_key_bytes() / 4;
    k_iks_key<kPksChunks, kPksNTiles, kPksWordsOut, kPksK>
        <<<(unsigned)((units + 255) / 256), 256, 0, st>>>(key_dev, key_tiles);
    return cudaGetLastError();
}

cudaError_t launch_privks_tc(const uint64_t* tlwe, int units, const uint8_t* key_tiles,
                             const PksMap& map, uint32_t* out, IksWorkspace& w, int* err,
                             cudaStream_t st, int* launches, bool prep)
{
    *launches = 0;
    if (units <= 0) return cudaSuccess;
    cudaError_t e = iks_tc_workspace(w, units, kPksChunks, st);
    constexpr int kMT = 2;  // two unit tiles per CTA share each 2.5 GB key's chunks
    if (e == cudaSuccess) e = gemm_attr<kPksChunks, kPksNTiles, kPksWordsOut, kMT>();
    if (e != cudaSuccess) return e;
    if (prep) k_pks_prep<<<units, 256, 0, st>>>(tlwe, units, map, w.atiles);
    const int gtiles = (units + kMGates - 1) / kMGates;
    const int ggroups = (gtiles + kMT - 1) / kMT;
    const OutMap om = {nullptr, map.per, map.stride_lo, map.stride_hi};
    k_iks_gemm<kPksChunks, kPksNTiles, kPksWordsOut, kMT>
        <<<ggroups * kPksNTiles, 128, iks_smem<kMT>(), st>>>(w.atiles, key_tiles, nullptr, nullptr,
                                                             units, out, om, err);
    *launches = prep ? 2 : 1;
    return cudaGetLastError();
}

}  // namespace cufhe
