// cufhe_gate_batch_noalloc: the batched gate path without any device
// allocation.
//
// Who needs it.  The regular batch entry point grows a per-stream workspace
// with cudaMalloc the first time a batch is larger than any before, and
// waits for the stream before it does so.  Some callers cannot let a library
// do that: a service that fixes its device-memory budget when it starts and
// treats any later allocation as a fault, a host program whose own allocator
// owns all device memory, or code on a latency-critical path that cannot
// absorb the device-wide synchronisation an allocation may bring.  For them
// this entry point keeps its lane buffers in one fixed array compiled into
// the library instead.
//
// What it costs.  The array below lives on every GPU that loads this
// library, from load until the process exits (kNoAllocBytes, about 1.7 MB),
// and limits one call to kNoAllocMaxLanes blind rotations.
//
// Sharing.  All calls on a device use the same array, and it keeps whatever
// the previous call left in it.  Every word a call reads from it is written
// earlier in the same call (key switching or pre-add fills the lvl0 lanes,
// blind rotation fills the lvl1 lanes), so nothing has to be cleared first.
// Two calls whose work overlaps on the GPU -- on different streams, or from
// different host threads -- race on the array and corrupt each other's
// results; order them on one stream or synchronise in between.
//
// Set-up.  Host code cannot take the address of a __device__ array
// directly: the array's name in host code is only a host-side handle, and a
// kernel given that handle would read the wrong memory or fault.  The first
// call on each device therefore asks the runtime for the array's device
// address (cudaGetSymbolAddress, with that device current) and caches it;
// that first call on a device should come before any stream capture.
#include <stdio.h>

#include "cufhe_b200.h"
#include "engine.h"

namespace cufhe {

namespace {

constexpr int kNoAllocMaxLanes = 256;
constexpr size_t kLaneInWords = (size_t)kNoAllocMaxLanes * kTlwe0;
constexpr size_t kLaneOutWords = (size_t)kNoAllocMaxLanes * kTlwe1;
constexpr size_t kNoAllocBytes = (kLaneInWords + kLaneOutWords) * sizeof(uint32_t);

// lanes' lvl0 inputs (first kLaneInWords words), then their lvl1 outputs
static __device__ __align__(256) uint32_t g_noalloc_scratch[kLaneInWords + kLaneOutWords];

constexpr int kMaxDevices = 16;
uint32_t* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (set-up on the
// first call per device).
int scratch_address(int device, uint32_t** out)
{
    if (device < 0 || device >= kMaxDevices)
        return engine_fail(CUFHE_ERR_ARG, "cufhe_gate_batch_noalloc: device index out of range");
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            char msg[256];
            snprintf(msg, sizeof(msg),
                     "cufhe_gate_batch_noalloc: cudaGetSymbolAddress of the scratch array "
                     "failed: %s", cudaGetErrorString(e));
            return engine_fail(CUFHE_ERR_CUDA, msg);
        }
        g_scratch_addr[device] = static_cast<uint32_t*>(p);
    }
    *out = g_scratch_addr[device];
    return CUFHE_OK;
}

int cuda_fail(const char* what, cudaError_t e)
{
    char msg[256];
    snprintf(msg, sizeof(msg), "cufhe_gate_batch_noalloc: %s: %s", what, cudaGetErrorString(e));
    return engine_fail(CUFHE_ERR_CUDA, msg);
}

}  // namespace

}  // namespace cufhe

using namespace cufhe;

extern "C" int cufhe_gate_batch_noalloc(int gate, size_t count, int level, uint32_t* out,
                                        const uint32_t* in0, const uint32_t* in1,
                                        const uint32_t* in2, cufhe_stream_t st)
{
    if (gate < 0 || gate >= kNumGates)
        return engine_fail(CUFHE_ERR_ARG, "cufhe_gate_batch_noalloc: bad gate id");
    if (level != CUFHE_LVL0 && level != CUFHE_LVL1)
        return engine_fail(CUFHE_ERR_ARG, "cufhe_gate_batch_noalloc: bad level");
    if (count == 0) return CUFHE_OK;
    const size_t lanes = count * (size_t)lanes_of_gate(gate);
    if (count > (size_t)kNoAllocMaxLanes || lanes > (size_t)kNoAllocMaxLanes) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "cufhe_gate_batch_noalloc: %zu gates need %zu blind rotations; at most %d "
                 "fit in its fixed scratch array (use cufhe_gate_batch for larger batches)",
                 count, lanes, kNoAllocMaxLanes);
        return engine_fail(CUFHE_ERR_ARG, msg);
    }
    if (!out || !in0 || (lanes && !in1) || ((gate == kMux || gate == kNMux) && !in2))
        return engine_fail(CUFHE_ERR_ARG, "cufhe_gate_batch_noalloc: missing operand");

    EngineView v;
    int rc = engine_view(st, &v);
    if (rc) return rc;
    cudaError_t e = cudaSetDevice(v.device);
    if (e != cudaSuccess) return cuda_fail("cudaSetDevice", e);
    uint32_t* scratch = nullptr;
    rc = scratch_address(v.device, &scratch);
    if (rc) return rc;
    uint32_t* lane_in = scratch;
    uint32_t* lane_out = scratch + kLaneInWords;

    Plan plan = Plan();
    plan.count = (int)count;
    plan.lanes = (int)lanes;
    plan.uniform_op = gate;  // uniform batch: lanes map arithmetically, no plan arrays

    int n = 0;
    if (lanes) {
        e = level == CUFHE_LVL1
                ? launch_iks(0, plan, in0, in1, in2, nullptr, v.ksk, lane_in, v.stream)
                : launch_preadd_lvl0(plan, in0, in1, in2, lane_in, v.stream);
        if (e != cudaSuccess) return cuda_fail("lane preparation", e);
        n++;
        e = launch_br_fp64(v.keybundle != 0, lane_in, (int)lanes, kMu, v.bkf, v.tables, -1,
                           nullptr, lane_out, v.stream);
        if (e != cudaSuccess) return cuda_fail("blind rotation", e);
        n++;
        e = level == CUFHE_LVL1
                ? launch_finalize_lvl1(plan, lane_out, out, v.stream)
                : launch_iks(1, plan, nullptr, nullptr, nullptr, lane_out, v.ksk, out, v.stream);
        if (e != cudaSuccess) return cuda_fail("gate outputs", e);
        n++;
    } else {
        e = launch_not_copy(plan, level == CUFHE_LVL1 ? kTlwe1 : kTlwe0, in0, out, v.stream);
        if (e != cudaSuccess) return cuda_fail("not/copy", e);
        n++;
    }
    engine_count_launches(n);
    return CUFHE_OK;
}
