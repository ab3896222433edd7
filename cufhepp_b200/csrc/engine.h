// Internal declarations shared by the engine's CUDA sources.
//
// Execution model.  A call of the gate API carries a batch of B gates.  Each
// gate expands into "lanes", one per blind rotation it needs: a binary gate
// has one lane, Mux/NMux have two (src/bootstrap_gpu.cu:1557-1672), Not/Copy
// none (:2200-2222).  Every kernel processes lanes or gates in bulk:
//
//   IKS->BR order (Ctxt<lvl1>):  k_iks (gate inputs -> lane lvl0 TLWEs)
//                                k_br_*  (lane lvl0 -> lane lvl1 TLWE, SE fused)
//                                k_finalize_lvl1 (lanes -> gate outputs)
//   BR->IKS order (Ctxt<lvl0>):  k_preadd_lvl0 (gate inputs -> lane lvl0)
//                                k_br_*
//                                k_iks (lanes combined -> gate outputs)
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <atomic>

#include "params.h"

namespace cufhe {

// "Function attribute already set on this device" flags of one kernel.
// cudaFuncSetAttribute acts on the current device only, so each device needs
// its own flag; the bits are atomic because several host threads may launch
// on different devices at once (setting an attribute twice is harmless).
class DeviceAttrFlags {
  public:
    bool test(int dev) const { return (bits_.load(std::memory_order_acquire) >> (dev & 63)) & 1u; }
    void set(int dev) { bits_.fetch_or(uint64_t(1) << (dev & 63), std::memory_order_release); }

  private:
    std::atomic<uint64_t> bits_{0};
};

// Sets the dynamic shared-memory limit of `func` on the current device once.
template <typename F>
cudaError_t set_smem_attr_once(DeviceAttrFlags& flags, F* func, size_t bytes)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (flags.test(dev)) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) flags.set(dev);
    return e;
}

constexpr int kN0 = CUFHE_LVL0_N;          // 636
constexpr int kN = CUFHE_LVL1_N;           // 1024
constexpr int kTlwe0 = CUFHE_TLWE0_WORDS;  // 637
constexpr int kTlwe1 = CUFHE_TLWE1_WORDS;  // 1025
constexpr int kTrlwe = CUFHE_TRLWE1_WORDS; // 2048
constexpr uint32_t kMu = CUFHE_MU32;

enum GateId {
    kNand = 0, kOr, kOrYN, kOrNY, kAnd, kAndYN, kAndNY, kNor, kXor, kXnor,
    kNot, kCopy, kMux, kNMux, kNumGates
};

// Pre-add coefficients of the binary gates, in the input level's torus
// (src/bootstrap_gpu.cu:1905-1914, :1937-1946).
struct GateCoef {
    int32_t ca, cb;
    uint32_t off;
};

__host__ __device__ inline GateCoef gate_coef(int g)
{
    const uint32_t mu = kMu;
    switch (g) {
    case kNand: return {-1, -1, mu};
    case kNor: return {-1, -1, 0u - mu};
    case kXnor: return {-2, -2, 0u - 2 * mu};
    case kAnd: return {1, 1, 0u - mu};
    case kOr: return {1, 1, mu};
    case kXor: return {2, 2, 2 * mu};
    case kAndNY: return {-1, 1, 0u - mu};
    case kAndYN: return {1, -1, 0u - mu};
    case kOrNY: return {-1, 1, mu};
    case kOrYN: return {1, -1, mu};
    default: return {1, 0, 0};
    }
}

__host__ __device__ inline int lanes_of_gate(int g)
{
    return (g == kMux || g == kNMux) ? 2 : (g == kNot || g == kCopy) ? 0 : 1;
}

// Lane plan of a batch.  With ops == nullptr every gate is `uniform_op` and
// lanes map arithmetically; otherwise lane_gate[l] is the gate of lane l,
// lane_sub[l] its index within the gate (0/1), gate_lane0[b] the first lane
// of gate b (-1 for Not/Copy).  Gate b reads operand k from row in_idx[k][b]
// of its input array and writes its result to row out_idx[b] of the output
// array (a circuit's wire table); a null index array means row b.
struct Plan {
    int count;       // gates
    int lanes;       // lanes
    int uniform_op;  // used when ops == nullptr
    const int8_t* ops;
    const int32_t* lane_gate;
    const int8_t* lane_sub;
    const int32_t* gate_lane0;
    const int32_t* in_idx[3];
    const int32_t* out_idx;
};

__device__ inline int plan_op(const Plan& p, int b) { return p.ops ? p.ops[b] : p.uniform_op; }

__device__ inline void plan_lane(const Plan& p, int l, int& b, int& sub)
{
    if (p.ops) {
        b = p.lane_gate[l];
        sub = p.lane_sub[l];
    } else if (lanes_of_gate(p.uniform_op) == 2) {
        b = l >> 1;
        sub = l & 1;
    } else {
        b = l;
        sub = 0;
    }
}

__host__ __device__ inline size_t plan_in_row(const Plan& p, int k, int b)
{
    return p.in_idx[k] ? (size_t)p.in_idx[k][b] : (size_t)b;
}

__host__ __device__ inline size_t plan_out_row(const Plan& p, int b)
{
    return p.out_idx ? (size_t)p.out_idx[b] : (size_t)b;
}

__device__ inline int plan_lane0(const Plan& p, int b)
{
    if (p.ops) return p.gate_lane0[b];
    const int n = lanes_of_gate(p.uniform_op);
    return n ? b * n : -1;
}

// Pre-add of lane (b, sub): x = ca * A + cb * B (+ off on b)
//   binary gate : A = in0[b], B = in1[b], table coefficients
//   mux lane 0  : A = inc = in0[b], B = in1[b], (1, 1, -mu)
//   mux lane 1  : A = inc = in0[b], B = in0_mux = in2[b], (-1, 1, -mu)
struct LanePreadd {
    const uint32_t* a;
    const uint32_t* b;
    int32_t ca, cb;
    uint32_t off;
};

__device__ inline LanePreadd lane_preadd(int op, int sub, const uint32_t* in0,
                                         const uint32_t* in1, const uint32_t* in2)
{
    if (op == kMux || op == kNMux) {
        if (sub == 0) return {in0, in1, 1, 1, 0u - kMu};
        return {in0, in2, -1, 1, 0u - kMu};
    }
    const GateCoef c = gate_coef(op);
    return {in0, in1, c.ca, c.cb, c.off};
}

// Pre-add of lane l of the plan from gate inputs of `words` words each
__device__ inline LanePreadd plan_lane_preadd(const Plan& p, int l, const uint32_t* in0,
                                              const uint32_t* in1, const uint32_t* in2, int words)
{
    int b, sub;
    plan_lane(p, l, b, sub);
    return lane_preadd(plan_op(p, b), sub, in0 + plan_in_row(p, 0, b) * words,
                       in1 ? in1 + plan_in_row(p, 1, b) * words : nullptr,
                       in2 ? in2 + plan_in_row(p, 2, b) * words : nullptr);
}

// Combination of a gate's lane outputs (lvl1 TLWEs) into the gate's lvl1
// result: binary -> lane0; Mux -> lane0 + lane1 + mu; NMux -> -(..) - mu.
__device__ inline LanePreadd gate_combine(int op, const uint32_t* lane0, const uint32_t* lane1)
{
    if (op == kMux) return {lane0, lane1, 1, 1, kMu};
    if (op == kNMux) return {lane0, lane1, -1, -1, 0u - kMu};
    return {lane0, nullptr, 1, 0, 0};
}

// ------------------------------------------------------------ launchers ----
// Each returns cudaSuccess or the launch error.

// IKS of lanes (mode 0: IKS->BR, gate inputs at lvl1 -> lane_in) or of gates
// (mode 1: BR->IKS, combined lane outputs -> out at lvl0).
cudaError_t launch_iks(int mode, const Plan& plan, const uint32_t* in0, const uint32_t* in1,
                       const uint32_t* in2, const uint32_t* lane_out, const uint32_t* ksk,
                       uint32_t* dst, cudaStream_t st);

cudaError_t launch_preadd_lvl0(const Plan& plan, const uint32_t* in0, const uint32_t* in1,
                               const uint32_t* in2, uint32_t* lane_in, cudaStream_t st);

cudaError_t launch_finalize_lvl1(const Plan& plan, const uint32_t* lane_out, uint32_t* out,
                                 cudaStream_t st);

cudaError_t launch_not_copy(const Plan& plan, int words, const uint32_t* in0, uint32_t* out,
                            cudaStream_t st);
// rows[0..nrows) of the wire table src copied into dst (same rows); dst may
// be a peer device's memory (peer access enabled)
cudaError_t launch_copy_rows(const int32_t* rows, int nrows, int words, const uint32_t* src,
                             uint32_t* dst, cudaStream_t st);

// FP64 FFNT blind rotation + SampleExtract of `lanes` lvl0 TLWEs.
// acc_out (optional) receives the TRLWE accumulators; lane_out (optional) the
// extracted lvl1 TLWEs.  steps < 0: all steps.
struct Fp64Tables {
    const double2* psi;    // psi^t, t < 2048, psi = e^{i pi / 1024}
    const double2* tw512;  // [16][32] e^{2 pi i n1 k2 / 512}
};
cudaError_t launch_br_fp64(bool kb, const uint32_t* lane_in, int lanes, uint32_t mu,
                           const double2* bkf, const Fp64Tables& t, int steps,
                           uint32_t* acc_out, uint32_t* lane_out, cudaStream_t st);

cudaError_t launch_bk_to_fft(const uint32_t* bk, int npolys, const Fp64Tables& t, double2* out,
                             cudaStream_t st);
// The same rotation with a fixed number of lanes per CTA (1, 2 or 4), for the
// autotuner; launch_br_fp64 picks it from the tuned table of the device
// (br_fp64_set_tuning) or, without one, from the batch size.
cudaError_t launch_br_fp64_g(int g, bool kb, const uint32_t* lane_in, int lanes, uint32_t mu,
                             const double2* bkf, const Fp64Tables& t, int steps,
                             uint32_t* acc_out, uint32_t* lane_out, cudaStream_t st);
// tuned choice for device dev: lanes <= bound[i] (ascending) -> g[i]; the last
// entry covers larger batches.  n = 0 clears the table.
void br_fp64_set_tuning(int dev, int n, const int* bound, const int* g);
int br_fp64_get_tuning(int dev, int* bound, int* g, int cap);
cudaError_t upload_fft_constants(void);

// Tensor-core identity key switching (iks_tc.cu).  Key tiles are built once
// per device from the raw KSK; the workspace holds per-batch one-hot digit
// tiles.  A timed-out device wait sets *err (checked at synchronisation).
struct IksWorkspace {
    size_t cap = 0;  // units
    int chunks = 0;  // K chunks per unit the tiles were sized for
    uint8_t* atiles = nullptr;
    uint32_t* xb = nullptr;
    int* valid = nullptr;
};
size_t iks_tc_key_bytes();
cudaError_t iks_tc_key_build(const uint32_t* ksk_dev, uint8_t* key_tiles, cudaStream_t st);
void iks_tc_workspace_free(IksWorkspace& w);
// sizes the workspace for `units` key switches up front (lvl1 or lvl2 inputs),
// so that later launches allocate nothing; a new workspace is zeroed on `st`
cudaError_t iks_tc_reserve(IksWorkspace& w, int units, bool lvl2, cudaStream_t st);
cudaError_t launch_iks_tc(int mode, const Plan& plan, const uint32_t* in0, const uint32_t* in1,
                          const uint32_t* in2, const uint32_t* lane_out, const uint8_t* key_tiles,
                          uint32_t* dst, IksWorkspace& w, int* err, cudaStream_t st,
                          int* launches);

// ------------------------------------------------ lvl0 -> lvl2 path ----
// psi2^s for s in [0, 512], psi2 = e^{i pi / 2048}: the root table of the
// N = 2048 transforms (other powers by symmetry)
constexpr int kPsi2Entries = 514;  // 513 used, padded to an even count

// FP64 FFNT blind rotation to lvl2 + SampleExtract of `lanes` lvl0 TLWEs;
// acc_out: TRLWE<lvl2> [lanes][4096], lane_out: TLWE<lvl2> [lanes][2049]
// (both optional, uint64 words).  bkf: Fourier BK [step][(e)][8][2][1024].
// in_count > 0: lane l rotates input l mod in_count with test value
// mu >> (mu_shift (l div in_count)) (several test polynomials in one launch)
cudaError_t launch_br2_fp64(bool kb, const uint32_t* lane_in, int lanes, uint64_t mu,
                            const double2* bkf, const double2* psi2, int steps, uint64_t* acc_out,
                            uint64_t* lane_out, cudaStream_t st, int in_count = 0,
                            int mu_shift = 0);
cudaError_t launch_bk2_to_fft(const uint64_t* bk, int npolys, const double2* psi2, double2* out,
                              cudaStream_t st);
cudaError_t upload_fft2_constants(void);

// Tensor-core key switching lvl2 -> lvl0 of gates (lane outputs at lvl2
// combined per gate: Mux +mu2, NMux negated -mu2) or, with plan.uniform_op a
// binary gate and no ops, of plain TLWE<lvl2> inputs.
size_t iks20_tc_key_bytes();
cudaError_t iks20_tc_key_build(const uint32_t* ksk_dev, uint8_t* key_tiles, cudaStream_t st);
cudaError_t launch_iks20_tc(const Plan& plan, const uint64_t* lane_out, const uint8_t* key_tiles,
                            uint32_t* dst, IksWorkspace& w, int* err, cudaStream_t st,
                            int* launches);

// ------------------------------- circuit bootstrapping, CMUX, lookup tables ----
// Private key switching TLWE<lvl2> -> TRLWE<lvl1>: unit u reads TLWE u (with
// badd[u / per] added to its b) and writes its TRLWE at
// out + (u % per) * stride_lo + (u / per) * stride_hi (words).
struct PksMap {
    int per;
    size_t stride_lo, stride_hi;
    uint64_t badd[4];
};
// on the tensor cores (iks_tc.cu): key tiles built once from the raw key
// [2049][10][15][2][1024]; the workspace holds the per-call one-hot tiles,
// which depend on the inputs only: prep = false reuses those of the previous
// call on the same inputs (the second key function of circuit bootstrapping)
size_t privks_tc_key_bytes();
cudaError_t privks_tc_key_build(const uint32_t* key_dev, uint8_t* key_tiles, cudaStream_t st);
cudaError_t launch_privks_tc(const uint64_t* tlwe, int units, const uint8_t* key_tiles,
                             const PksMap& map, uint32_t* out, IksWorkspace& w, int* err,
                             cudaStream_t st, int* launches, bool prep = true);

// Batched CMUX: CMUX c = (g, m) with g = c / per, m = c % per reads d0/d1 at
// node g * node_stride_g + m * node_stride_m (TRLWE units), the Fourier TRGSW at
// trgsw + g * trgsw_stride (double2 units) and writes out[g * per + m].
struct CmuxPlan {
    int count, per;
    size_t node_stride_g, node_stride_m;
    const uint32_t* d0;
    const uint32_t* d1;
    const double2* trgsw;
    size_t trgsw_stride;
    uint32_t* out;
};
cudaError_t launch_cmux(int gadget, const CmuxPlan& p, const Fp64Tables& t, cudaStream_t st);
cudaError_t launch_lut_leaves(const uint8_t* luts, int q, uint32_t mu, uint32_t* nodes,
                              cudaStream_t st);
cudaError_t launch_extract8(const uint32_t* roots, int q, uint32_t* out, cudaStream_t st);
cudaError_t upload_cb_constants(void);
// a one-thread kernel whose bounded mbarrier wait (polls tries) runs out and
// sets *err like the tensor-core kernels do
cudaError_t launch_wait_timeout_probe(int* err, uint32_t polls, cudaStream_t st);

// Read-only view of the engine state that a gate call on stream `st` uses
// (keys of the stream's device and the CUDA stream).  Returns 0 or a
// CUFHE_ERR_* code (and sets the last error).
struct EngineView {
    int device;
    cudaStream_t stream;
    int keybundle;
    const uint32_t* ksk;
    const double2* bkf;
    Fp64Tables tables;
};
int engine_view(void* st, EngineView* v);
// sets the message returned by cufhe_last_error() and returns code
int engine_fail(int code, const char* msg);
// counts kernel launches reported by cufhe_kernel_launches()
void engine_count_launches(int n);

}  // namespace cufhe
