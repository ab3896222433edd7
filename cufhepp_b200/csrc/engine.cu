// C-ABI of the gate engine (include/cufhe_b200.h): global key state per GPU,
// streams with their own workspaces, and the batched gate pipeline.
//
// Reference counterparts: Initialize/CleanUp (src/cufhe_gates_gpu.cu:34-73),
// key uploads (src/keyswitch_gpu.cu:7-22, src/bootstrap_gpu.cu:212-332), FFT
// tables (src/ntt_small_modulus.cu:207-244, :369-443), Stream / StreamQuery /
// Synchronize (include/cufhe_gpu.cuh:70-76, :162-199), gate entry points
// (src/cufhe_gates_gpu.cu:198-824).
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <vector>

#include "cufhe_b200.h"
#include "engine.h"
#include "br_int8.h"

namespace cufhe {

namespace {

constexpr int kMaxDev = 16;

struct DeviceState {
    bool ready = false;
    int kb = 0;
    uint32_t* ksk = nullptr;
    double2* bkf = nullptr;  // FP64 Fourier-domain bootstrapping key
    double2* psi = nullptr;
    double2* tw512 = nullptr;
    Int8Key i8;              // INT8 exact-path key (plain or KeyBundle, as the FP64 one)
    Int8Key i8_2;            // INT8 exact-path lvl02 key (plain or KeyBundle)
    uint8_t* iks_key = nullptr;  // KSK as signed byte-limb tiles (tensor-core IKS)
    int* err = nullptr;          // set by a device wait that timed out
    // lvl0 -> lvl2 path (Initialize_lvl02)
    bool ready2 = false;
    int kb2 = 0;
    double2* bkf2 = nullptr;     // FP64 Fourier-domain BK<lvl2>
    double2* psi2 = nullptr;     // psi2^s, s <= 512
    uint8_t* iks2_key = nullptr; // lvl20 KSK byte-limb tiles
    int* err2 = nullptr;
    // circuit bootstrapping (cufhe_initialize_cb)
    bool ready_cb = false;
    uint8_t* pks[2] = {nullptr, nullptr};   // private key-switching keys lvl2 -> lvl1 (limb tiles)
    int* err_cb = nullptr;
    double2* cb_psi = nullptr;               // lvl1 FFT tables for CMUX
    double2* cb_tw512 = nullptr;
};

struct Workspace {
    size_t lane_cap = 0, gate_cap = 0, io_cap = 0, stage_cap = 0;
    uint32_t* lane_in = nullptr;
    uint32_t* lane_out = nullptr;
    int8_t* ops = nullptr;
    int32_t* lane_gate = nullptr;
    int8_t* lane_sub = nullptr;
    int32_t* gate_lane0 = nullptr;
    uint32_t* io = nullptr;  // device staging for batch_host: in0,in1,in2,out
    unsigned char* stage = nullptr;  // pinned host staging for plan uploads
    cudaEvent_t stage_ev = nullptr;
    Int8Workspace i8;
    Int8Workspace2 i8_2;
    IksWorkspace iks;
    size_t lane2_cap = 0;
    uint64_t* lane_out2 = nullptr;  // lvl2 lane outputs [lanes][2049]
    IksWorkspace iks2;
    size_t lut_cap = 0;             // lookup tables the node buffers hold
    uint32_t* lut_a = nullptr;      // CMUX-tree node buffers [q][256] / [q][128] TRLWEs
    uint32_t* lut_b = nullptr;
    uint8_t* lut_tab = nullptr;     // the tables, [q][256] bytes
    IksWorkspace iks_pks;           // one-hot tiles of the private key switch
};

}  // namespace
}  // namespace cufhe

struct cufhe_stream_s {
    cudaStream_t st = nullptr;
    int device = 0;
    cufhe::Workspace ws;
};

// A levelised gate circuit (cufhe_circuit_create): one Plan per wave of
// independent gates, all plan and index arrays in one device buffer, and a
// private workspace sized for the widest wave, so that running the circuit
// allocates nothing and can be captured into a CUDA graph.
struct cufhe_circuit_s {
    int device = 0;
    int level = 0;
    size_t wires = 0, gates = 0;
    int max_lanes = 0, max_gates = 0;
    std::vector<cufhe::Plan> waves;
    std::vector<char> wave_nc;  // wave holds Not/Copy gates
    void* dbuf = nullptr;
    cufhe_stream_s exec;        // workspace of the circuit; exec.st = the stream of a run
    cudaStream_t cap = nullptr; // private stream the graph is captured on
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    uint32_t* graph_wires = nullptr;
    int graph_precision = -1;
    uint64_t graph_launches = 0;
    // cufhe_circuit_create_split: groups of the circuit's connected components,
    // each a circuit of its own (waves, workspace, graph) run on its own
    // stream, all groups concurrently; the fields above are then unused
    std::vector<cufhe_circuit_s*> parts;
    std::vector<cudaStream_t> part_st;
    std::vector<cudaEvent_t> part_done;
    cudaEvent_t part_fork = nullptr;
};

namespace cufhe {
namespace {

int g_gpu_num = 1;
int g_stream_count = 0;
int g_precision = CUFHE_FP64_FFNT;
DeviceState g_dev[kMaxDev];
cufhe_stream_s g_default[kMaxDev];
char g_err[512] = "";
std::atomic<uint64_t> g_launches{0};

// optional per-kernel-class event timing (cufhe_profile_*)
struct ProfRec {
    cudaEvent_t a, b;
    int cls;
};
bool g_prof = false;
std::vector<ProfRec> g_prof_recs;
double g_prof_ms[CUFHE_K_CLASSES] = {};
uint64_t g_prof_n[CUFHE_K_CLASSES] = {};

void prof_begin(cudaStream_t st, ProfRec& r, int cls)
{
    r.cls = cls;
    r.a = r.b = nullptr;
    if (!g_prof) return;
    cudaEventCreate(&r.a);
    cudaEventCreate(&r.b);
    cudaEventRecord(r.a, st);
}

void prof_end(cudaStream_t st, ProfRec& r)
{
    if (!r.a) return;
    cudaEventRecord(r.b, st);
    g_prof_recs.push_back(r);
}

int fail(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(CUFHE_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                             \
    } while (0)

#define CKL(call)              \
    do {                       \
        CK(call);              \
        g_launches.fetch_add(1); \
    } while (0)

// launch one engine kernel of class `cls` on stream `st` (timed when profiling)
#define LAUNCH(cls, st, call)      \
    do {                           \
        ProfRec pr_;               \
        prof_begin((st), pr_, (cls)); \
        CKL(call);                 \
        prof_end((st), pr_);       \
    } while (0)

void free_ws(Workspace& w)
{
    cudaFree(w.lane_in);
    cudaFree(w.lane_out);
    cudaFree(w.ops);
    cudaFree(w.lane_gate);
    cudaFree(w.lane_sub);
    cudaFree(w.gate_lane0);
    cudaFree(w.io);
    if (w.stage) cudaFreeHost(w.stage);
    if (w.stage_ev) cudaEventDestroy(w.stage_ev);
    int8_workspace_free(w.i8);
    int8_workspace2_free(w.i8_2);
    iks_tc_workspace_free(w.iks);
    cudaFree(w.lane_out2);
    iks_tc_workspace_free(w.iks2);
    cudaFree(w.lut_a);
    cudaFree(w.lut_b);
    cudaFree(w.lut_tab);
    iks_tc_workspace_free(w.iks_pks);
    w = Workspace();
}

// grow workspace buffers; waits for the stream first so no kernel still uses
// the old ones
int ensure_ws(cufhe_stream_s* s, size_t gates, size_t lanes)
{
    Workspace& w = s->ws;
    if (lanes > w.lane_cap) {
        CK(cudaStreamSynchronize(s->st));
        cudaFree(w.lane_in);
        cudaFree(w.lane_out);
        cudaFree(w.lane_gate);
        cudaFree(w.lane_sub);
        w.lane_in = w.lane_out = nullptr;
        size_t cap = lanes < 256 ? 256 : lanes;
        CK(cudaMalloc(&w.lane_in, cap * kTlwe0 * sizeof(uint32_t)));
        CK(cudaMalloc(&w.lane_out, cap * kTlwe1 * sizeof(uint32_t)));
        CK(cudaMalloc(&w.lane_gate, cap * sizeof(int32_t)));
        CK(cudaMalloc(&w.lane_sub, cap));
        w.lane_cap = cap;
    }
    if (gates > w.gate_cap) {
        CK(cudaStreamSynchronize(s->st));
        cudaFree(w.ops);
        cudaFree(w.gate_lane0);
        size_t cap = gates < 256 ? 256 : gates;
        CK(cudaMalloc(&w.ops, cap));
        CK(cudaMalloc(&w.gate_lane0, cap * sizeof(int32_t)));
        w.gate_cap = cap;
    }
    return CUFHE_OK;
}

cufhe_stream_s* resolve(cufhe_stream_t st)
{
    if (st) return st;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxDev) dev = 0;
    g_default[dev].device = dev;
    return &g_default[dev];
}

void host_tables(std::vector<double2>& psi, std::vector<double2>& tw)
{
    const long double pi = 3.141592653589793238462643383279502884L;
    psi.resize(2 * kN);
    for (int t = 0; t < 2 * kN; t++) {
        const long double a = pi * t / kN;  // psi = e^{i pi / N}
        psi[t] = make_double2((double)cosl(a), (double)sinl(a));
    }
    tw.resize(16 * 32);
    for (int k2 = 0; k2 < 16; k2++)
        for (int n1 = 0; n1 < 32; n1++) {
            const long double a = 2 * pi * (long double)(n1 * k2) / 512;
            tw[k2 * 32 + n1] = make_double2((double)cosl(a), (double)sinl(a));
        }
}

void release_cb(int d);

void release_device02(int d)
{
    DeviceState& D = g_dev[d];
    cudaSetDevice(d);
    release_cb(d);
    cudaFree(D.bkf2);
    cudaFree(D.psi2);
    cudaFree(D.iks2_key);
    cudaFree(D.err2);
    int8_key_free(D.i8_2);
    D.bkf2 = D.psi2 = nullptr;
    D.iks2_key = nullptr;
    D.err2 = nullptr;
    D.ready2 = false;
    D.kb2 = 0;
}

void release_cb(int d)
{
    DeviceState& D = g_dev[d];
    cudaSetDevice(d);
    cudaFree(D.pks[0]);
    cudaFree(D.pks[1]);
    cudaFree(D.cb_psi);
    cudaFree(D.cb_tw512);
    cudaFree(D.err_cb);
    D.err_cb = nullptr;
    D.pks[0] = D.pks[1] = nullptr;
    D.cb_psi = D.cb_tw512 = nullptr;
    D.ready_cb = false;
}

void release_device(int d)
{
    DeviceState& D = g_dev[d];
    cudaSetDevice(d);
    release_cb(d);
    release_device02(d);
    cudaFree(D.ksk);
    cudaFree(D.bkf);
    cudaFree(D.psi);
    cudaFree(D.tw512);
    cudaFree(D.iks_key);
    cudaFree(D.err);
    int8_key_free(D.i8);
    D = DeviceState();
    free_ws(g_default[d].ws);
}

int init_device(int d, const cufhe_keyview* ek)
{
    DeviceState& D = g_dev[d];
    CK(cudaSetDevice(d));
    CK(upload_fft_constants());
    std::vector<double2> psi, tw;
    host_tables(psi, tw);
    CK(cudaMalloc(&D.psi, psi.size() * sizeof(double2)));
    CK(cudaMalloc(&D.tw512, tw.size() * sizeof(double2)));
    CK(cudaMemcpy(D.psi, psi.data(), psi.size() * sizeof(double2), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(D.tw512, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice));

    CK(cudaMalloc(&D.ksk, ek->ksk_words * sizeof(uint32_t)));
    CK(cudaMemcpy(D.ksk, ek->ksk, ek->ksk_words * sizeof(uint32_t), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&D.iks_key, iks_tc_key_bytes()));
    CKL(iks_tc_key_build(D.ksk, D.iks_key, 0));
    CK(cudaMalloc(&D.err, sizeof(int)));
    CK(cudaMemset(D.err, 0, sizeof(int)));

    uint32_t* raw = nullptr;
    CK(cudaMalloc(&raw, ek->bk_words * sizeof(uint32_t)));
    CK(cudaMemcpy(raw, ek->bk, ek->bk_words * sizeof(uint32_t), cudaMemcpyHostToDevice));
    const int npolys = (int)(ek->bk_words / kN);
    CK(cudaMalloc(&D.bkf, (size_t)npolys * 512 * sizeof(double2)));
    const Fp64Tables t = {D.psi, D.tw512};
    CKL(launch_bk_to_fft(raw, npolys, t, D.bkf, 0));
    {
        // INT8 Toeplitz limb windows of either key form (KeyBundle: 954 TRGSWs)
        cudaError_t e = int8_key_build(D.i8, raw, ek->keybundle != 0, 0);
        if (e != cudaSuccess) {
            cudaFree(raw);
            return fail(CUFHE_ERR_CUDA, "INT8 key conversion: %s", cudaGetErrorString(e));
        }
    }
    CK(cudaDeviceSynchronize());
    cudaFree(raw);
    D.kb = ek->keybundle;
    D.ready = true;
    return CUFHE_OK;
}

// Initialize_lvl02 on device d (src/cufhe_gates_gpu.cu:75-90): FFT tables of
// N = 2048, Fourier BK<lvl2>, lvl20 key tiles
int init_device02(int d, const cufhe_keyview02* ek)
{
    DeviceState& D = g_dev[d];
    CK(cudaSetDevice(d));
    CK(upload_fft2_constants());
    std::vector<double2> tab(kPsi2Entries, make_double2(0.0, 0.0));
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int t = 0; t <= 512; t++) {
        const long double a = pi * t / CUFHE_LVL2_N;
        tab[t] = make_double2((double)cosl(a), (double)sinl(a));
    }
    CK(cudaMalloc(&D.psi2, tab.size() * sizeof(double2)));
    CK(cudaMemcpy(D.psi2, tab.data(), tab.size() * sizeof(double2), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&D.err2, sizeof(int)));
    CK(cudaMemset(D.err2, 0, sizeof(int)));

    uint32_t* ksk = nullptr;
    CK(cudaMalloc(&ksk, ek->ksk_words * sizeof(uint32_t)));
    CK(cudaMemcpy(ksk, ek->ksk, ek->ksk_words * sizeof(uint32_t), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&D.iks2_key, iks20_tc_key_bytes()));
    CKL(iks20_tc_key_build(ksk, D.iks2_key, 0));

    uint64_t* raw = nullptr;
    CK(cudaMalloc(&raw, ek->bk_words * sizeof(uint64_t)));
    CK(cudaMemcpy(raw, ek->bk, ek->bk_words * sizeof(uint64_t), cudaMemcpyHostToDevice));
    const int npolys = (int)(ek->bk_words / CUFHE_LVL2_N);
    CK(cudaMalloc(&D.bkf2, (size_t)npolys * 1024 * sizeof(double2)));
    CKL(launch_bk2_to_fft(raw, npolys, D.psi2, D.bkf2, 0));
    {
        // INT8 Toeplitz limb windows of either key form (KeyBundle: 954 TRGSWs)
        cudaError_t e = int8_key2_build(D.i8_2, raw, ek->keybundle != 0, 0);
        if (e != cudaSuccess) {
            cudaFree(raw);
            cudaFree(ksk);
            return fail(CUFHE_ERR_CUDA, "INT8 lvl02 key conversion: %s", cudaGetErrorString(e));
        }
    }
    CK(cudaDeviceSynchronize());
    cudaFree(raw);
    cudaFree(ksk);
    D.kb2 = ek->keybundle;
    D.ready2 = true;
    return CUFHE_OK;
}

// cufhe_initialize_cb on device d: private key-switching keys and the lvl1
// FFT tables of the CMUX kernels
int init_cb(int d, const cufhe_cbkeyview* kv)
{
    DeviceState& D = g_dev[d];
    CK(cudaSetDevice(d));
    CK(upload_cb_constants());
    CK(upload_fft_constants());  // k_bk_to_fft (TRGSW -> Fourier) lives in br_fp64.cu
    std::vector<double2> psi, tw;
    host_tables(psi, tw);
    CK(cudaMalloc(&D.cb_psi, psi.size() * sizeof(double2)));
    CK(cudaMalloc(&D.cb_tw512, tw.size() * sizeof(double2)));
    CK(cudaMemcpy(D.cb_psi, psi.data(), psi.size() * sizeof(double2), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(D.cb_tw512, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&D.err_cb, sizeof(int)));
    CK(cudaMemset(D.err_cb, 0, sizeof(int)));
    const uint32_t* src[2] = {kv->privks0, kv->privks1};
    uint32_t* raw = nullptr;
    if (cudaMalloc(&raw, kv->words * sizeof(uint32_t)) != cudaSuccess)
        return fail(CUFHE_ERR_NOMEM, "private key-switching key (%zu words)", kv->words);
    for (int f = 0; f < 2; f++) {
        cudaError_t e = cudaMalloc(&D.pks[f], privks_tc_key_bytes());
        if (e == cudaSuccess)
            e = cudaMemcpy(raw, src[f], kv->words * sizeof(uint32_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = privks_tc_key_build(raw, D.pks[f], 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            cudaFree(raw);
            return fail(CUFHE_ERR_CUDA, "private key-switching key tiles: %s", cudaGetErrorString(e));
        }
        g_launches.fetch_add(1);
    }
    cudaFree(raw);
    D.ready_cb = true;
    return CUFHE_OK;
}

// Host-side lane plan of a batch (uploaded through pinned staging).
int build_plan(cufhe_stream_s* s, const int32_t* gates, int uniform, size_t count, Plan& plan)
{
    plan = Plan();
    plan.count = (int)count;
    plan.uniform_op = uniform;
    if (!gates) {
        if (uniform < 0 || uniform >= kNumGates) return fail(CUFHE_ERR_ARG, "bad gate id %d", uniform);
        plan.lanes = (int)(count * lanes_of_gate(uniform));
        return ensure_ws(s, count, plan.lanes);
    }
    size_t lanes = 0;
    for (size_t b = 0; b < count; b++) {
        if (gates[b] < 0 || gates[b] >= kNumGates)
            return fail(CUFHE_ERR_ARG, "bad gate id %d at %zu", gates[b], b);
        lanes += lanes_of_gate(gates[b]);
    }
    int rc = ensure_ws(s, count, lanes);
    if (rc) return rc;
    Workspace& w = s->ws;
    const size_t bytes = count * (1 + 4) + lanes * (4 + 1);
    if (bytes > w.stage_cap) {
        if (w.stage) {
            CK(cudaEventSynchronize(w.stage_ev));
            cudaFreeHost(w.stage);
            w.stage = nullptr;
        }
        CK(cudaMallocHost(&w.stage, bytes));
        if (!w.stage_ev) CK(cudaEventCreateWithFlags(&w.stage_ev, cudaEventDisableTiming));
        w.stage_cap = bytes;
    } else if (w.stage_ev) {
        CK(cudaEventSynchronize(w.stage_ev));  // previous upload finished reading
    }
    int8_t* ops = (int8_t*)w.stage;
    int32_t* g0 = (int32_t*)(w.stage + count);
    int32_t* lg = (int32_t*)(w.stage + count * 5);
    int8_t* ls = (int8_t*)(w.stage + count * 5 + lanes * 4);
    size_t l = 0;
    for (size_t b = 0; b < count; b++) {
        const int n = lanes_of_gate(gates[b]);
        ops[b] = (int8_t)gates[b];
        g0[b] = n ? (int32_t)l : -1;
        for (int k = 0; k < n; k++, l++) {
            lg[l] = (int32_t)b;
            ls[l] = (int8_t)k;
        }
    }
    CK(cudaMemcpyAsync(w.ops, ops, count, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(w.gate_lane0, g0, count * 4, cudaMemcpyHostToDevice, s->st));
    if (lanes) {
        CK(cudaMemcpyAsync(w.lane_gate, lg, lanes * 4, cudaMemcpyHostToDevice, s->st));
        CK(cudaMemcpyAsync(w.lane_sub, ls, lanes, cudaMemcpyHostToDevice, s->st));
    }
    CK(cudaEventRecord(w.stage_ev, s->st));
    plan.lanes = (int)lanes;
    plan.ops = w.ops;
    plan.lane_gate = w.lane_gate;
    plan.lane_sub = w.lane_sub;
    plan.gate_lane0 = w.gate_lane0;
    return CUFHE_OK;
}

// identity key switching of lanes (mode 0) or gates (mode 1) on the tensor cores
int run_iks(cufhe_stream_s* s, int mode, const Plan& plan, const uint32_t* in0, const uint32_t* in1,
            const uint32_t* in2, const uint32_t* lane_out, uint32_t* dst)
{
    DeviceState& D = g_dev[s->device];
    int launches = 0;
    ProfRec pr;
    prof_begin(s->st, pr, CUFHE_K_IKS);
    cudaError_t e = launch_iks_tc(mode, plan, in0, in1, in2, lane_out, D.iks_key, dst, s->ws.iks,
                                  D.err, s->st, &launches);
    prof_end(s->st, pr);
    g_launches.fetch_add(launches);
    if (e != cudaSuccess) return fail(CUFHE_ERR_CUDA, "key switching: %s", cudaGetErrorString(e));
    return CUFHE_OK;
}

// reports (and clears) a device-side wait timeout recorded on device d
int check_device_error(int d)
{
    DeviceState& D = g_dev[d];
    int* flags[3] = {D.ready ? D.err : nullptr, D.ready2 ? D.err2 : nullptr,
                     D.ready_cb ? D.err_cb : nullptr};
    for (int* f : flags) {
        if (!f) continue;
        int h = 0;
        CK(cudaMemcpy(&h, f, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) {
            cudaMemset(f, 0, sizeof(int));
            return fail(CUFHE_ERR_CUDA, "a tensor-core kernel's bounded wait timed out (code %d)", h);
        }
    }
    return CUFHE_OK;
}

// private key switching lvl2 -> lvl1 on the tensor cores
int run_privks(cufhe_stream_s* s, const uint64_t* tlwe2, int units, int func, const PksMap& map,
               uint32_t* out, bool prep = true)
{
    DeviceState& D = g_dev[s->device];
    int launches = 0;
    ProfRec pr;
    prof_begin(s->st, pr, CUFHE_K_PRIVKS);
    cudaError_t e = launch_privks_tc(tlwe2, units, D.pks[func], map, out, s->ws.iks_pks, D.err_cb,
                                     s->st, &launches, prep);
    prof_end(s->st, pr);
    g_launches.fetch_add(launches);
    if (e != cudaSuccess) return fail(CUFHE_ERR_CUDA, "private key switching: %s", cudaGetErrorString(e));
    return CUFHE_OK;
}

// lvl2 -> lvl0 key switching of gates on the tensor cores
int run_iks20(cufhe_stream_s* s, const Plan& plan, const uint64_t* lane_out, uint32_t* dst)
{
    DeviceState& D = g_dev[s->device];
    int launches = 0;
    ProfRec pr;
    prof_begin(s->st, pr, CUFHE_K_IKS_LVL20);
    cudaError_t e = launch_iks20_tc(plan, lane_out, D.iks2_key, dst, s->ws.iks2, D.err2, s->st,
                                    &launches);
    prof_end(s->st, pr);
    g_launches.fetch_add(launches);
    if (e != cudaSuccess) return fail(CUFHE_ERR_CUDA, "lvl20 key switching: %s", cudaGetErrorString(e));
    return CUFHE_OK;
}

// in_count > 0 (FP64 form only): lane l rotates input l mod in_count with
// test value mu >> (mu_shift (l div in_count))
int run_br2(cufhe_stream_s* s, const uint32_t* lane_in, int lanes, uint64_t mu, int steps,
            uint64_t* acc_out, uint64_t* lane_out, int in_count = 0, int mu_shift = 0)
{
    DeviceState& D = g_dev[s->device];
    if (g_precision == CUFHE_INT8_EXACT) {
        if (!D.i8_2.ready) return fail(CUFHE_ERR_STATE, "INT8_EXACT: no lvl02 INT8 key on this device");
        int launches = 0;
        ProfRec pr;
        prof_begin(s->st, pr, CUFHE_K_BR_INT8_LVL02);
        cudaError_t e = launch_br2_int8(D.i8_2, s->ws.i8_2, lane_in, lanes, mu, steps, acc_out,
                                        lane_out, D.err2, s->st, &launches);
        prof_end(s->st, pr);
        g_launches.fetch_add(launches);
        if (e != cudaSuccess)
            return fail(CUFHE_ERR_CUDA, "INT8 lvl02 blind rotation: %s", cudaGetErrorString(e));
        return CUFHE_OK;
    }
    LAUNCH(CUFHE_K_BR_FP64_LVL02, s->st,
           launch_br2_fp64(D.kb2 != 0, lane_in, lanes, mu, D.bkf2, D.psi2, steps, acc_out, lane_out,
                           s->st, in_count, mu_shift));
    return CUFHE_OK;
}

int ensure_lane2(cufhe_stream_s* s, size_t lanes)
{
    Workspace& w = s->ws;
    if (lanes <= w.lane2_cap) return CUFHE_OK;
    CK(cudaStreamSynchronize(s->st));
    cudaFree(w.lane_out2);
    w.lane_out2 = nullptr;
    const size_t cap = lanes < 256 ? 256 : lanes;
    if (cudaMalloc(&w.lane_out2, cap * CUFHE_TLWE2_WORDS * sizeof(uint64_t)) != cudaSuccess)
        return fail(CUFHE_ERR_NOMEM, "lvl2 lane buffer for %zu lanes", cap);
    w.lane2_cap = cap;
    return CUFHE_OK;
}

// blind rotation of plan.lanes lanes with the selected precision form
int run_br(cufhe_stream_s* s, const uint32_t* lane_in, int lanes, uint32_t mu, int steps,
           uint32_t* acc_out, uint32_t* lane_out)
{
    DeviceState& D = g_dev[s->device];
    if (g_precision == CUFHE_INT8_EXACT) {
        if (!D.i8.ready) return fail(CUFHE_ERR_STATE, "INT8_EXACT: no INT8 key on this device");
        int launches = 0;
        ProfRec pr;
        prof_begin(s->st, pr, CUFHE_K_BR_INT8);
        cudaError_t e = launch_br_int8(D.i8, s->ws.i8, lane_in, lanes, mu, steps, acc_out,
                                       lane_out, D.err, s->st, &launches);
        prof_end(s->st, pr);
        g_launches.fetch_add(launches);
        if (e != cudaSuccess) return fail(CUFHE_ERR_CUDA, "INT8 blind rotation: %s", cudaGetErrorString(e));
        return CUFHE_OK;
    }
    const Fp64Tables t = {D.psi, D.tw512};
    LAUNCH(CUFHE_K_BR_FP64, s->st,
           launch_br_fp64(D.kb != 0, lane_in, lanes, mu, D.bkf, t, steps, acc_out, lane_out, s->st));
    return CUFHE_OK;
}

int run_batch(cufhe_stream_s* s, const int32_t* gates, int uniform, size_t count, int level,
              uint32_t* out, const uint32_t* in0, const uint32_t* in1, const uint32_t* in2)
{
    if (level != CUFHE_LVL0 && level != CUFHE_LVL1 && level != CUFHE_LVL02)
        return fail(CUFHE_ERR_ARG, "bad level %d", level);
    if (count == 0) return CUFHE_OK;
    if (count > (1u << 24)) return fail(CUFHE_ERR_ARG, "batch of %zu gates too large", count);
    if (!out || !in0) return fail(CUFHE_ERR_ARG, "null ciphertext pointer");
    bool need1 = false, need2 = false;
    if (gates) {
        for (size_t b = 0; b < count; b++) {
            need1 |= lanes_of_gate(gates[b]) > 0;
            need2 |= gates[b] == kMux || gates[b] == kNMux;
        }
    } else {
        need1 = lanes_of_gate(uniform) > 0;
        need2 = uniform == kMux || uniform == kNMux;
    }
    if ((need1 && !in1) || (need2 && !in2)) return fail(CUFHE_ERR_ARG, "missing input operand");
    // keys are needed by gates that bootstrap; Not/Copy alone run without them
    // (the reference's lvl02 test runs Not/Copy<lvl0param> after Initialize_lvl02 only)
    if (need1 && (level == CUFHE_LVL02 ? !g_dev[s->device].ready2 : !g_dev[s->device].ready))
        return fail(CUFHE_ERR_STATE, level == CUFHE_LVL02 ? "cufhe_initialize_lvl02() not called"
                                                         : "cufhe_initialize() not called");
    CK(cudaSetDevice(s->device));
    Plan plan;
    int rc = build_plan(s, gates, uniform, count, plan);
    if (rc) return rc;
    Workspace& w = s->ws;
    if (plan.lanes && level == CUFHE_LVL02) {
        // *_lvl02 gates: lvl0 pre-add, blind rotation to lvl2, combination +
        // key switching lvl2 -> lvl0 (src/cufhe_gates_gpu.cu:826-979)
        rc = ensure_lane2(s, plan.lanes);
        if (rc) return rc;
        LAUNCH(CUFHE_K_PREADD, s->st, launch_preadd_lvl0(plan, in0, in1, in2, w.lane_in, s->st));
        rc = run_br2(s, w.lane_in, plan.lanes, CUFHE_MU64, -1, nullptr, w.lane_out2);
        if (rc) return rc;
        rc = run_iks20(s, plan, w.lane_out2, out);
        if (rc) return rc;
    } else if (plan.lanes) {
        if (level == CUFHE_LVL1) {
            rc = run_iks(s, 0, plan, in0, in1, in2, nullptr, w.lane_in);
            if (rc) return rc;
        } else
            LAUNCH(CUFHE_K_PREADD, s->st, launch_preadd_lvl0(plan, in0, in1, in2, w.lane_in, s->st));
        rc = run_br(s, w.lane_in, plan.lanes, kMu, -1, nullptr, w.lane_out);
        if (rc) return rc;
        if (level == CUFHE_LVL1) {
            LAUNCH(CUFHE_K_FINALIZE, s->st, launch_finalize_lvl1(plan, w.lane_out, out, s->st));
        } else {
            rc = run_iks(s, 1, plan, nullptr, nullptr, nullptr, w.lane_out, out);
            if (rc) return rc;
        }
    }
    const bool any_nc = gates ? true : (uniform == kNot || uniform == kCopy);
    if (any_nc) {
        bool has = !gates;
        for (size_t b = 0; gates && b < count && !has; b++)
            has = gates[b] == kNot || gates[b] == kCopy;
        if (has)
            LAUNCH(CUFHE_K_FINALIZE, s->st,
                   launch_not_copy(plan, level == CUFHE_LVL1 ? kTlwe1 : kTlwe0, in0, out, s->st));
    // (lvl02 gates keep Ctxt<lvl0> I/O, so Not/Copy work on TLWE<lvl0> there too)
    }
    return CUFHE_OK;
}

// ------------------------------------------------------------ circuits ----
// Runs wave w of circuit c on the wire table `wires` on stream c->exec.st.
int run_wave(cufhe_circuit_s* c, size_t w, uint32_t* wires)
{
    const Plan& plan = c->waves[w];
    cufhe_stream_s* s = &c->exec;
    Workspace& ws = s->ws;
    int rc = CUFHE_OK;
    if (plan.lanes) {
        if (c->level == CUFHE_LVL1) {
            if ((rc = run_iks(s, 0, plan, wires, wires, wires, nullptr, ws.lane_in))) return rc;
            if ((rc = run_br(s, ws.lane_in, plan.lanes, kMu, -1, nullptr, ws.lane_out))) return rc;
            LAUNCH(CUFHE_K_FINALIZE, s->st, launch_finalize_lvl1(plan, ws.lane_out, wires, s->st));
        } else if (c->level == CUFHE_LVL0) {
            LAUNCH(CUFHE_K_PREADD, s->st,
                   launch_preadd_lvl0(plan, wires, wires, wires, ws.lane_in, s->st));
            if ((rc = run_br(s, ws.lane_in, plan.lanes, kMu, -1, nullptr, ws.lane_out))) return rc;
            if ((rc = run_iks(s, 1, plan, nullptr, nullptr, nullptr, ws.lane_out, wires))) return rc;
        } else {
            LAUNCH(CUFHE_K_PREADD, s->st,
                   launch_preadd_lvl0(plan, wires, wires, wires, ws.lane_in, s->st));
            if ((rc = run_br2(s, ws.lane_in, plan.lanes, CUFHE_MU64, -1, nullptr, ws.lane_out2)))
                return rc;
            if ((rc = run_iks20(s, plan, ws.lane_out2, wires))) return rc;
        }
    }
    if (c->wave_nc[w])
        LAUNCH(CUFHE_K_FINALIZE, s->st,
               launch_not_copy(plan, c->level == CUFHE_LVL1 ? kTlwe1 : kTlwe0, wires, wires, s->st));
    return CUFHE_OK;
}

void circuit_drop_graph(cufhe_circuit_s* c)
{
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->gexec = nullptr;
    c->graph = nullptr;
    c->graph_wires = nullptr;
}

// Captures every wave into a CUDA graph (on the circuit's private stream);
// `st` is the stream the graph is launched on next
int circuit_capture(cufhe_circuit_s* c, uint32_t* wires, cudaStream_t st)
{
    circuit_drop_graph(c);
    if (g_precision == CUFHE_INT8_EXACT && c->max_lanes > 0) {
        // the INT8 workspace must not be allocated inside the capture; a new
        // one is zeroed on `st`, ahead of the graph launch
        const cudaError_t e = c->level == CUFHE_LVL02
                                  ? int8_reserve2(c->exec.ws.i8_2, c->max_lanes, st)
                                  : int8_reserve(c->exec.ws.i8, c->max_lanes, st);
        if (e != cudaSuccess)
            return fail(CUFHE_ERR_NOMEM, "INT8 workspace: %s", cudaGetErrorString(e));
    }
    const bool prof = g_prof;
    g_prof = false;  // per-kernel event timing is not recorded inside graphs
    const uint64_t l0 = g_launches.load();
    CK(cudaStreamBeginCapture(c->cap, cudaStreamCaptureModeRelaxed));
    c->exec.st = c->cap;
    int rc = CUFHE_OK;
    for (size_t w = 0; w < c->waves.size() && !rc; w++) rc = run_wave(c, w, wires);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->cap, &g);
    g_prof = prof;
    c->graph_launches = g_launches.load() - l0;
    g_launches.fetch_sub(c->graph_launches);  // counted when the graph runs
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(CUFHE_ERR_CUDA, "circuit capture: %s", cudaGetErrorString(e));
    c->graph = g;
    CK(cudaGraphInstantiate(&c->gexec, g, 0));
    c->graph_wires = wires;
    c->graph_precision = g_precision;
    return CUFHE_OK;
}

void circuit_free(cufhe_circuit_s* c)
{
    cudaSetDevice(c->device);
    for (cufhe_circuit_s* q : c->parts) circuit_free(q);
    for (cudaStream_t st : c->part_st) cudaStreamDestroy(st);
    for (cudaEvent_t ev : c->part_done) cudaEventDestroy(ev);
    if (c->part_fork) cudaEventDestroy(c->part_fork);
    circuit_drop_graph(c);
    cudaFree(c->dbuf);
    free_ws(c->exec.ws);
    if (c->cap) cudaStreamDestroy(c->cap);
    delete c;
}

// lanes per CTA of the FP64 blind rotation measured on the current device for a
// ladder of batch sizes (the autotuner behind cufhe_autotune)
int autotune_br(int d)
{
    DeviceState& D = g_dev[d];
    if (!D.ready) return fail(CUFHE_ERR_STATE, "cufhe_initialize() not called");
    int sms = 148;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d));
    const int ladder[] = {1, sms / 2, sms, 2 * sms, 3 * sms, 4 * sms, 6 * sms, 8 * sms,
                          12 * sms, 16 * sms, 24 * sms, 32 * sms};
    const int n = (int)(sizeof(ladder) / sizeof(ladder[0]));
    const int maxl = ladder[n - 1];
    uint32_t *lin = nullptr, *lout = nullptr;
    CK(cudaMalloc(&lin, (size_t)maxl * kTlwe0 * 4));
    if (cudaMalloc(&lout, (size_t)maxl * kTlwe1 * 4) != cudaSuccess) {
        cudaFree(lin);
        return fail(CUFHE_ERR_NOMEM, "autotune buffers");
    }
    cudaMemset(lin, 0, (size_t)maxl * kTlwe0 * 4);  // valid (noiseless zero) inputs
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const Fp64Tables t = {D.psi, D.tw512};
    int bound[32], best[32];
    int rc = CUFHE_OK;
    for (int i = 0; i < n && !rc; i++) {
        const int L = ladder[i];
        float best_ms = 1e30f;
        best[i] = 1;
        bound[i] = L;
        const int cands[] = {1, 2, 4};
        for (int g : cands) {
            float ms_min = 1e30f;
            for (int rep = 0; rep < 3; rep++) {
                cudaEventRecord(e0, 0);
                cudaError_t e = launch_br_fp64_g(g, D.kb != 0, lin, L, kMu, D.bkf, t, -1, nullptr,
                                                 lout, 0);
                cudaEventRecord(e1, 0);
                if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                if (e != cudaSuccess) {
                    rc = fail(CUFHE_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
                    break;
                }
                g_launches.fetch_add(1);
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0 && ms < ms_min) ms_min = ms;  // first run warms up
            }
            if (rc) break;
            if (ms_min < best_ms * 0.98f) {  // prefer fewer lanes per CTA on a tie
                best_ms = ms_min;
                best[i] = g;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(lin);
    cudaFree(lout);
    if (!rc) br_fp64_set_tuning(d, n, bound, best);
    return rc;
}

}  // namespace

int engine_view(void* st, EngineView* v)
{
    cufhe_stream_s* s = resolve(static_cast<cufhe_stream_t>(st));
    const DeviceState& D = g_dev[s->device];
    if (!D.ready) return fail(CUFHE_ERR_STATE, "cufhe_initialize() not called");
    v->device = s->device;
    v->stream = s->st;
    v->keybundle = D.kb;
    v->ksk = D.ksk;
    v->bkf = D.bkf;
    v->tables = {D.psi, D.tw512};
    return CUFHE_OK;
}

int engine_fail(int code, const char* msg) { return fail(code, "%s", msg); }

void engine_count_launches(int n) { g_launches.fetch_add(n); }

}  // namespace cufhe

using namespace cufhe;

extern "C" {

int cufhe_set_gpu_num(int n)
{
    int avail = 0;
    if (cudaGetDeviceCount(&avail) != cudaSuccess) avail = 0;
    if (n < 1 || n > kMaxDev) return fail(CUFHE_ERR_ARG, "gpu num %d out of range", n);
    if (avail && n > avail) return fail(CUFHE_ERR_ARG, "only %d GPUs visible", avail);
    g_gpu_num = n;
    return CUFHE_OK;
}

int cufhe_get_gpu_num(void) { return g_gpu_num; }

int cufhe_initialize(const cufhe_keyview* ek)
{
    if (!ek || !ek->bk || !ek->ksk) return fail(CUFHE_ERR_ARG, "null key view");
    const uint64_t want_bk = ek->keybundle ? CUFHE_BKKB1_WORDS : CUFHE_BK1_WORDS;
    if (ek->bk_words != want_bk)
        return fail(CUFHE_ERR_ARG, "bootstrapping key has %zu words, expected %llu", ek->bk_words,
                    (unsigned long long)want_bk);
    if (ek->ksk_words != CUFHE_KSK10_WORDS)
        return fail(CUFHE_ERR_ARG, "key-switching key has %zu words, expected %llu",
                    ek->ksk_words, (unsigned long long)CUFHE_KSK10_WORDS);
    int avail = 0;
    if (cudaGetDeviceCount(&avail) != cudaSuccess || avail == 0)
        return fail(CUFHE_ERR_CUDA, "no CUDA device visible");
    if (g_gpu_num > avail) return fail(CUFHE_ERR_ARG, "gpu num %d > %d visible", g_gpu_num, avail);
    for (int d = 0; d < g_gpu_num; d++) {
        if (g_dev[d].ready) release_device(d);
        int rc = init_device(d, ek);
        if (rc) {
            release_device(d);
            return rc;
        }
    }
    cudaSetDevice(0);
    return CUFHE_OK;
}

// engine streams of cufhe_gate_batch_sharded_host, one per shard
static std::vector<cufhe_stream_t> g_shard_st;

static void release_shard_streams()
{
    for (cufhe_stream_t st : g_shard_st) cufhe_stream_destroy(st);
    g_shard_st.clear();
}

int cufhe_cleanup(void)
{
    release_shard_streams();
    for (int d = 0; d < kMaxDev; d++)
        if (g_dev[d].ready) release_device(d);
    cudaSetDevice(0);
    return CUFHE_OK;
}

int cufhe_initialize_lvl02(const cufhe_keyview02* ek)
{
    if (!ek || !ek->bk || !ek->ksk) return fail(CUFHE_ERR_ARG, "null key view");
    const uint64_t want_bk = ek->keybundle ? CUFHE_BKKB2_WORDS : CUFHE_BK2_WORDS;
    if (ek->bk_words != want_bk)
        return fail(CUFHE_ERR_ARG, "lvl02 bootstrapping key has %zu words, expected %llu",
                    ek->bk_words, (unsigned long long)want_bk);
    if (ek->ksk_words != CUFHE_KSK20_WORDS)
        return fail(CUFHE_ERR_ARG, "lvl20 key-switching key has %zu words, expected %llu",
                    ek->ksk_words, (unsigned long long)CUFHE_KSK20_WORDS);
    int avail = 0;
    if (cudaGetDeviceCount(&avail) != cudaSuccess || avail == 0)
        return fail(CUFHE_ERR_CUDA, "no CUDA device visible");
    if (g_gpu_num > avail) return fail(CUFHE_ERR_ARG, "gpu num %d > %d visible", g_gpu_num, avail);
    for (int d = 0; d < g_gpu_num; d++) {
        if (g_dev[d].ready2) release_device02(d);
        int rc = init_device02(d, ek);
        if (rc) {
            release_device02(d);
            return rc;
        }
    }
    cudaSetDevice(0);
    return CUFHE_OK;
}

int cufhe_cleanup_lvl02(void)
{
    for (int d = 0; d < kMaxDev; d++)
        if (g_dev[d].ready2) release_device02(d);
    cudaSetDevice(0);
    return CUFHE_OK;
}

int cufhe_selftest_wait_timeout(void)
{
    cufhe_stream_s* s = resolve(nullptr);
    DeviceState& D = g_dev[s->device];
    if (!D.ready) return fail(CUFHE_ERR_STATE, "cufhe_initialize() not called");
    CK(cudaSetDevice(s->device));
    CKL(launch_wait_timeout_probe(D.err, 1u << 14, s->st));
    CK(cudaStreamSynchronize(s->st));
    return check_device_error(s->device);
}

int cufhe_synchronize(void)
{
    for (int d = 0; d < g_gpu_num; d++) {
        CK(cudaSetDevice(d));
        CK(cudaDeviceSynchronize());
        const int rc = check_device_error(d);
        if (rc) return rc;
    }
    return CUFHE_OK;
}

int cufhe_set_precision(int form)
{
    if (form != CUFHE_FP64_FFNT && form != CUFHE_INT8_EXACT)
        return fail(CUFHE_ERR_ARG, "unknown precision form %d", form);
    g_precision = form;
    return CUFHE_OK;
}

int cufhe_get_precision(void) { return g_precision; }

int cufhe_stream_create(cufhe_stream_t* st, int device)
{
    if (!st) return fail(CUFHE_ERR_ARG, "null stream handle");
    if (device < 0) device = g_stream_count % g_gpu_num;
    if (device >= g_gpu_num) return fail(CUFHE_ERR_ARG, "device %d >= gpu num", device);
    g_stream_count++;
    cufhe_stream_s* s = new cufhe_stream_s();
    s->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete s;
        return fail(CUFHE_ERR_CUDA, "stream create: %s", cudaGetErrorString(e));
    }
    *st = s;
    return CUFHE_OK;
}

int cufhe_stream_destroy(cufhe_stream_t st)
{
    if (!st) return CUFHE_OK;
    cudaSetDevice(st->device);
    cudaStreamSynchronize(st->st);
    free_ws(st->ws);
    cudaStreamDestroy(st->st);
    delete st;
    return CUFHE_OK;
}

int cufhe_stream_query(cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    cudaSetDevice(s->device);
    cudaError_t e = cudaStreamQuery(s->st);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) return 0;
    return fail(CUFHE_ERR_CUDA, "stream query: %s", cudaGetErrorString(e));
}

int cufhe_stream_device(cufhe_stream_t st) { return resolve(st)->device; }

int cufhe_stream_cuda(cufhe_stream_t st, void** cuda_stream)
{
    if (!cuda_stream) return fail(CUFHE_ERR_ARG, "null pointer");
    *cuda_stream = static_cast<void*>(resolve(st)->st);
    return CUFHE_OK;
}

int cufhe_stream_synchronize(cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->st));
    return check_device_error(s->device);
}

int cufhe_ctxt_alloc(void** dptr, size_t bytes, int device)
{
    if (!dptr) return fail(CUFHE_ERR_ARG, "null pointer");
    CK(cudaSetDevice(device < 0 ? 0 : device));
    if (cudaMalloc(dptr, bytes) != cudaSuccess) return fail(CUFHE_ERR_NOMEM, "cudaMalloc(%zu) failed", bytes);
    return CUFHE_OK;
}

int cufhe_ctxt_free(void* dptr, int device)
{
    CK(cudaSetDevice(device < 0 ? 0 : device));
    CK(cudaFree(dptr));
    return CUFHE_OK;
}

int cufhe_host_register(void* host, size_t bytes)
{
    CK(cudaHostRegister(host, bytes, cudaHostRegisterDefault));
    return CUFHE_OK;
}

int cufhe_host_unregister(void* host)
{
    CK(cudaHostUnregister(host));
    return CUFHE_OK;
}

int cufhe_memcpy_h2d(void* dst, const void* src, size_t bytes, cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    CK(cudaSetDevice(s->device));
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->st));
    return CUFHE_OK;
}

int cufhe_memcpy_d2h(void* dst, const void* src, size_t bytes, cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    CK(cudaSetDevice(s->device));
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->st));
    return CUFHE_OK;
}

int cufhe_gate(int gate, int level, uint32_t* out, const uint32_t* in0, const uint32_t* in1,
               const uint32_t* in2, cufhe_stream_t st)
{
    if (gate < 0 || gate >= kNumGates) return fail(CUFHE_ERR_ARG, "bad gate id %d", gate);
    return run_batch(resolve(st), nullptr, gate, 1, level, out, in0, in1, in2);
}

int cufhe_gate_copy(int gate, int level, uint32_t* out_host, uint32_t* out_dev,
                    const uint32_t* in0_host, uint32_t* in0_dev, const uint32_t* in1_host,
                    uint32_t* in1_dev, const uint32_t* in2_host, uint32_t* in2_dev,
                    cufhe_stream_t st)
{
    if (gate < 0 || gate >= kNumGates) return fail(CUFHE_ERR_ARG, "bad gate id %d", gate);
    cufhe_stream_s* s = resolve(st);
    const size_t bytes = (level == CUFHE_LVL1 ? kTlwe1 : kTlwe0) * sizeof(uint32_t);
    CK(cudaSetDevice(s->device));
    const int nin = gate == kNot || gate == kCopy ? 1 : (gate == kMux || gate == kNMux ? 3 : 2);
    const uint32_t* hs[3] = {in0_host, in1_host, in2_host};
    uint32_t* ds[3] = {in0_dev, in1_dev, in2_dev};
    for (int i = 0; i < nin; i++) {
        if (!hs[i] || !ds[i]) return fail(CUFHE_ERR_ARG, "missing operand %d", i);
        CK(cudaMemcpyAsync(ds[i], hs[i], bytes, cudaMemcpyHostToDevice, s->st));
    }
    int rc = run_batch(s, nullptr, gate, 1, level, out_dev, in0_dev, in1_dev, in2_dev);
    if (rc) return rc;
    CK(cudaMemcpyAsync(out_host, out_dev, bytes, cudaMemcpyDeviceToHost, s->st));
    return CUFHE_OK;
}

int cufhe_gate_batch(const int32_t* gates_host, int uniform_gate, size_t count, int level,
                     uint32_t* out, const uint32_t* in0, const uint32_t* in1, const uint32_t* in2,
                     cufhe_stream_t st)
{
    return run_batch(resolve(st), gates_host, uniform_gate, count, level, out, in0, in1, in2);
}

int cufhe_gate_batch_host(const int32_t* gates_host, int uniform_gate, size_t count, int level,
                          uint32_t* out_host, const uint32_t* in0_host, const uint32_t* in1_host,
                          const uint32_t* in2_host, cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    if (count == 0) return CUFHE_OK;
    const size_t words = level == CUFHE_LVL1 ? kTlwe1 : kTlwe0;
    const size_t bytes = count * words * sizeof(uint32_t);
    CK(cudaSetDevice(s->device));
    Workspace& w = s->ws;
    if (4 * count * words > w.io_cap) {
        CK(cudaStreamSynchronize(s->st));
        cudaFree(w.io);
        w.io = nullptr;
        if (cudaMalloc(&w.io, 4 * bytes) != cudaSuccess)
            return fail(CUFHE_ERR_NOMEM, "io buffer of %zu bytes", 4 * bytes);
        w.io_cap = 4 * count * words;
    }
    uint32_t* d0 = w.io;
    uint32_t* d1 = w.io + count * words;
    uint32_t* d2 = w.io + 2 * count * words;
    uint32_t* dout = w.io + 3 * count * words;
    CK(cudaMemcpyAsync(d0, in0_host, bytes, cudaMemcpyHostToDevice, s->st));
    if (in1_host) CK(cudaMemcpyAsync(d1, in1_host, bytes, cudaMemcpyHostToDevice, s->st));
    if (in2_host) CK(cudaMemcpyAsync(d2, in2_host, bytes, cudaMemcpyHostToDevice, s->st));
    int rc = run_batch(s, gates_host, uniform_gate, count, level, dout, d0, in1_host ? d1 : nullptr,
                       in2_host ? d2 : nullptr);
    if (rc) return rc;
    CK(cudaMemcpyAsync(out_host, dout, bytes, cudaMemcpyDeviceToHost, s->st));
    return CUFHE_OK;
}

int cufhe_blind_rotate(const uint32_t* tlwe0, size_t count, uint32_t mu, int steps,
                       uint32_t* acc_out, uint32_t* tlwe_out, cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    if (!g_dev[s->device].ready) return fail(CUFHE_ERR_STATE, "cufhe_initialize() not called");
    if (!tlwe0 || (!acc_out && !tlwe_out)) return fail(CUFHE_ERR_ARG, "null pointer");
    if (count == 0) return CUFHE_OK;
    if (count > (1u << 24)) return fail(CUFHE_ERR_ARG, "too many inputs");
    CK(cudaSetDevice(s->device));
    return run_br(s, tlwe0, (int)count, mu, steps, acc_out, tlwe_out);
}

int cufhe_identity_keyswitch(const uint32_t* tlwe1, size_t count, uint32_t* tlwe0_out,
                             cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    if (!g_dev[s->device].ready) return fail(CUFHE_ERR_STATE, "cufhe_initialize() not called");
    if (!tlwe1 || !tlwe0_out) return fail(CUFHE_ERR_ARG, "null pointer");
    if (count == 0) return CUFHE_OK;
    if (count > (1u << 24)) return fail(CUFHE_ERR_ARG, "too many inputs");
    CK(cudaSetDevice(s->device));
    Plan plan = Plan();
    plan.count = plan.lanes = (int)count;
    // mode 1 reads the inputs as lane outputs; a binary gate id gives one lane
    // per input and the identity combination (1, 0, 0)
    plan.uniform_op = kAnd;
    return run_iks(s, 1, plan, nullptr, nullptr, nullptr, tlwe1, tlwe0_out);
}

int cufhe_blind_rotate_lvl02(const uint32_t* tlwe0, size_t count, uint64_t mu, int steps,
                             uint64_t* acc_out, uint64_t* tlwe2_out, cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    if (!g_dev[s->device].ready2) return fail(CUFHE_ERR_STATE, "cufhe_initialize_lvl02() not called");
    if (!tlwe0 || (!acc_out && !tlwe2_out)) return fail(CUFHE_ERR_ARG, "null pointer");
    if (count == 0) return CUFHE_OK;
    if (count > (1u << 24)) return fail(CUFHE_ERR_ARG, "too many inputs");
    CK(cudaSetDevice(s->device));
    return run_br2(s, tlwe0, (int)count, mu, steps, acc_out, tlwe2_out);
}

int cufhe_identity_keyswitch_lvl20(const uint64_t* tlwe2, size_t count, uint32_t* tlwe0_out,
                                   cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    if (!g_dev[s->device].ready2) return fail(CUFHE_ERR_STATE, "cufhe_initialize_lvl02() not called");
    if (!tlwe2 || !tlwe0_out) return fail(CUFHE_ERR_ARG, "null pointer");
    if (count == 0) return CUFHE_OK;
    if (count > (1u << 24)) return fail(CUFHE_ERR_ARG, "too many inputs");
    CK(cudaSetDevice(s->device));
    Plan plan = Plan();
    plan.count = plan.lanes = (int)count;
    plan.uniform_op = kAnd;  // one lane per input, identity combination
    return run_iks20(s, plan, tlwe2, tlwe0_out);
}

// Validation, levelisation and balancing of a circuit on the host (no GPU):
// wave[g] for every gate, nwaves = the critical path.  `sms` sets the
// balancing's round of lanes (4 x sms at lvl0/lvl1, 2 x sms at lvl02).
static int plan_waves(int level, size_t num_wires, size_t num_gates, const int32_t* gate_ops,
                      const int32_t* in0, const int32_t* in1, const int32_t* in2,
                      const int32_t* out, int sms, std::vector<int32_t>& wave, int& nwaves)
{
    if (level != CUFHE_LVL0 && level != CUFHE_LVL1 && level != CUFHE_LVL02)
        return fail(CUFHE_ERR_ARG, "bad level %d", level);
    if (num_gates == 0 || num_wires == 0) return fail(CUFHE_ERR_ARG, "empty circuit");
    if (num_gates > (1u << 26) || num_wires > (1u << 30))
        return fail(CUFHE_ERR_ARG, "circuit too large");
    if (!gate_ops || !in0 || !out) return fail(CUFHE_ERR_ARG, "null circuit array");
    if (sms <= 0) sms = 148;

    // ---- validation: gate ids, operand and result wires, single assignment
    std::vector<int32_t> producer(num_wires, -1);
    for (size_t g = 0; g < num_gates; g++) {
        const int op = gate_ops[g];
        if (op < 0 || op >= kNumGates) return fail(CUFHE_ERR_ARG, "bad gate id %d at gate %zu", op, g);
        const int nin = (op == kNot || op == kCopy) ? 1 : ((op == kMux || op == kNMux) ? 3 : 2);
        const int32_t* ins[3] = {in0, in1, in2};
        for (int k = 0; k < nin; k++) {
            if (!ins[k]) return fail(CUFHE_ERR_ARG, "gate %zu needs operand %d", g, k);
            if (ins[k][g] < 0 || (size_t)ins[k][g] >= num_wires)
                return fail(CUFHE_ERR_ARG, "gate %zu operand %d: wire %d out of range", g, k, ins[k][g]);
        }
        if (out[g] < 0 || (size_t)out[g] >= num_wires)
            return fail(CUFHE_ERR_ARG, "gate %zu result wire %d out of range", g, out[g]);
        if (producer[out[g]] >= 0)
            return fail(CUFHE_ERR_ARG, "wire %d is written by gates %d and %zu", out[g],
                        producer[out[g]], g);
        producer[out[g]] = (int32_t)g;
    }
    // ---- levelisation (Kahn): wave of a gate = 1 + latest wave of its producers
    std::vector<int32_t> indeg(num_gates, 0), head(num_gates, -1), nxt, to;
    wave.assign(num_gates, 0);
    for (size_t g = 0; g < num_gates; g++) {
        const int op = gate_ops[g];
        const int nin = (op == kNot || op == kCopy) ? 1 : ((op == kMux || op == kNMux) ? 3 : 2);
        const int32_t* ins[3] = {in0, in1, in2};
        for (int k = 0; k < nin; k++) {
            const int32_t p = producer[ins[k][g]];
            if (p < 0) continue;
            indeg[g]++;
            nxt.push_back(head[p]);
            to.push_back((int32_t)g);
            head[p] = (int32_t)(to.size() - 1);
        }
    }
    std::vector<int32_t> queue;
    queue.reserve(num_gates);
    for (size_t g = 0; g < num_gates; g++)
        if (!indeg[g]) queue.push_back((int32_t)g);
    for (size_t qi = 0; qi < queue.size(); qi++) {
        const int32_t g = queue[qi];
        for (int32_t e = head[g]; e >= 0; e = nxt[e]) {
            const int32_t h = to[e];
            if (wave[g] + 1 > wave[h]) wave[h] = wave[g] + 1;
            if (--indeg[h] == 0) queue.push_back(h);
        }
    }
    if (queue.size() != num_gates) return fail(CUFHE_ERR_ARG, "the circuit has a cycle");
    nwaves = 0;
    for (size_t g = 0; g < num_gates; g++) nwaves = wave[g] + 1 > nwaves ? wave[g] + 1 : nwaves;
    // ---- balancing: a wave of up to `cap` blind-rotation lanes costs one
    // rotation latency whatever its width, so gates with slack move out of
    // waves above `cap` into the latest later wave with room (never at or past
    // a consumer's wave).  Gates go in reverse topological order, so every
    // consumer's wave is final when its producer moves; the number of waves
    // stays the critical path.
    {
        const long cap = (long)(level == CUFHE_LVL02 ? 2 : 4) * sms;
        std::vector<long> load(nwaves, 0);
        for (size_t g = 0; g < num_gates; g++) load[wave[g]] += lanes_of_gate(gate_ops[g]);
        for (size_t qi = num_gates; qi-- > 0;) {
            const int32_t g = queue[qi];
            if (load[wave[g]] <= cap) continue;
            int maxw = nwaves - 1;
            for (int32_t e = head[g]; e >= 0; e = nxt[e])
                maxw = wave[to[e]] - 1 < maxw ? wave[to[e]] - 1 : maxw;
            const long lg = lanes_of_gate(gate_ops[g]);
            for (int w = maxw; w > wave[g]; w--)
                if (load[w] + lg <= cap) {
                    load[wave[g]] -= lg;
                    load[w] += lg;
                    wave[g] = w;
                    break;
                }
        }
    }
    return CUFHE_OK;
}

int cufhe_circuit_plan(int level, size_t num_wires, size_t num_gates, const int32_t* gate_ops,
                       const int32_t* in0, const int32_t* in1, const int32_t* in2,
                       const int32_t* out, int sms, int32_t* wave_of_gate, int* num_waves)
{
    if (!wave_of_gate || !num_waves) return fail(CUFHE_ERR_ARG, "null plan output");
    std::vector<int32_t> wave;
    int nwaves = 0;
    const int rc = plan_waves(level, num_wires, num_gates, gate_ops, in0, in1, in2, out, sms, wave,
                              nwaves);
    if (rc != CUFHE_OK) return rc;
    for (size_t g = 0; g < num_gates; g++) wave_of_gate[g] = wave[g];
    *num_waves = nwaves;
    return CUFHE_OK;
}

// Connected components of the gate graph (a gate is joined to the producers
// of its operands), packed into at most `parts` groups with balanced blind
// rotations: components by decreasing weight, each into the lightest group
// (weight = 16 x lanes + gates, so that Not/Copy-only components count too).
// Gates of different groups read no wire the other group writes, so the
// groups can run concurrently.  The circuit must be valid (plan_waves).
// Returns the number of non-empty groups, numbered 0 .. n-1.
static int split_components(size_t num_wires, size_t num_gates, const int32_t* gate_ops,
                            const int32_t* in0, const int32_t* in1, const int32_t* in2,
                            const int32_t* out, int parts, std::vector<int32_t>& group)
{
    std::vector<int32_t> parent(num_gates), producer(num_wires, -1);
    for (size_t g = 0; g < num_gates; g++) {
        parent[g] = (int32_t)g;
        producer[out[g]] = (int32_t)g;
    }
    auto find = [&](int32_t x) {
        while (parent[x] != x) {
            parent[x] = parent[parent[x]];
            x = parent[x];
        }
        return x;
    };
    for (size_t g = 0; g < num_gates; g++) {
        const int op = gate_ops[g];
        const int nin = (op == kNot || op == kCopy) ? 1 : ((op == kMux || op == kNMux) ? 3 : 2);
        const int32_t* ins[3] = {in0, in1, in2};
        for (int k = 0; k < nin; k++) {
            const int32_t q = producer[ins[k][g]];
            if (q < 0) continue;
            const int32_t a = find((int32_t)g), b = find(q);
            if (a != b) parent[a] = b;
        }
    }
    std::vector<int64_t> weight(num_gates, 0);
    for (size_t g = 0; g < num_gates; g++)
        weight[find((int32_t)g)] += 16 * lanes_of_gate(gate_ops[g]) + 1;
    std::vector<int32_t> comps;
    for (size_t g = 0; g < num_gates; g++)
        if (parent[g] == (int32_t)g) comps.push_back((int32_t)g);
    std::stable_sort(comps.begin(), comps.end(),
                     [&](int32_t a, int32_t b) { return weight[a] > weight[b]; });
    const int np = (int)std::min<size_t>((size_t)parts, comps.size());
    std::vector<int64_t> load(np, 0);
    std::vector<int32_t> group_of_root(num_gates, -1);
    for (int32_t r : comps) {
        int k = 0;
        for (int i = 1; i < np; i++)
            if (load[i] < load[k]) k = i;
        group_of_root[r] = k;
        load[k] += weight[r];
    }
    group.assign(num_gates, 0);
    for (size_t g = 0; g < num_gates; g++) group[g] = group_of_root[find((int32_t)g)];
    return np;
}

int cufhe_circuit_split_plan(int level, size_t num_wires, size_t num_gates,
                             const int32_t* gate_ops, const int32_t* in0, const int32_t* in1,
                             const int32_t* in2, const int32_t* out, int parts,
                             int32_t* group_of_gate)
{
    if (!group_of_gate) return fail(CUFHE_ERR_ARG, "null plan output");
    if (parts < 1 || parts > 64) return fail(CUFHE_ERR_ARG, "parts %d outside 1..64", parts);
    std::vector<int32_t> wave;
    int nwaves = 0;
    int rc = plan_waves(level, num_wires, num_gates, gate_ops, in0, in1, in2, out, 0, wave, nwaves);
    if (rc != CUFHE_OK) return rc;
    std::vector<int32_t> group;
    rc = split_components(num_wires, num_gates, gate_ops, in0, in1, in2, out, parts, group);
    for (size_t g = 0; g < num_gates; g++) group_of_gate[g] = group[g];
    return rc;
}

// Device form of a planned circuit: one Plan per wave over the gates
// members[w], packed into one device buffer, and a private workspace for the
// widest wave.  Waves may be empty (a shard of a sharded circuit).
static int build_circuit(cufhe_circuit_t* out_c, int level, size_t num_wires, size_t num_gates,
                         const int32_t* gate_ops, const int32_t* in0, const int32_t* in1,
                         const int32_t* in2, const int32_t* out, int device,
                         const std::vector<std::vector<int32_t>>& members)
{
    const int nwaves = (int)members.size();
    // ---- per-wave plan arrays, packed into one buffer (16-byte aligned)
    auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
    std::vector<size_t> off(nwaves);
    size_t total = 0;
    int max_lanes = 0, max_gates = 0;
    for (int w = 0; w < nwaves; w++) {
        const size_t n = members[w].size();
        size_t lanes = 0;
        for (int32_t g : members[w]) lanes += lanes_of_gate(gate_ops[g]);
        off[w] = total;
        total += al(n) + al(4 * n) + al(4 * lanes) + al(lanes) + 4 * al(4 * n);
        max_lanes = (int)lanes > max_lanes ? (int)lanes : max_lanes;
        max_gates = (int)n > max_gates ? (int)n : max_gates;
    }
    if (total == 0) total = 16;
    std::vector<unsigned char> host(total, 0);
    cufhe_circuit_s* c = new cufhe_circuit_s();
    c->device = device;
    c->level = level;
    c->wires = num_wires;
    c->gates = num_gates;
    c->max_lanes = max_lanes;
    c->max_gates = max_gates;
    c->exec.device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaMalloc(&c->dbuf, total);
    if (e != cudaSuccess) {
        circuit_free(c);
        return fail(CUFHE_ERR_NOMEM, "circuit plan buffer: %s", cudaGetErrorString(e));
    }
    unsigned char* dbase = static_cast<unsigned char*>(c->dbuf);
    for (int w = 0; w < nwaves; w++) {
        const std::vector<int32_t>& m = members[w];
        const size_t n = m.size();
        size_t lanes = 0;
        for (int32_t g : m) lanes += lanes_of_gate(gate_ops[g]);
        size_t o = off[w];
        const size_t o_ops = o; o += al(n);
        const size_t o_l0 = o; o += al(4 * n);
        const size_t o_lg = o; o += al(4 * lanes);
        const size_t o_ls = o; o += al(lanes);
        size_t o_idx[4];
        for (int k = 0; k < 4; k++) { o_idx[k] = o; o += al(4 * n); }
        int8_t* ops = (int8_t*)&host[o_ops];
        int32_t* l0 = (int32_t*)&host[o_l0];
        int32_t* lg = (int32_t*)&host[o_lg];
        int8_t* ls = (int8_t*)&host[o_ls];
        int32_t* idx[4];
        for (int k = 0; k < 4; k++) idx[k] = (int32_t*)&host[o_idx[k]];
        size_t l = 0;
        bool nc = false;
        for (size_t b = 0; b < n; b++) {
            const int32_t g = m[b];
            const int op = gate_ops[g];
            const int nl = lanes_of_gate(op);
            ops[b] = (int8_t)op;
            l0[b] = nl ? (int32_t)l : -1;
            for (int k = 0; k < nl; k++, l++) {
                lg[l] = (int32_t)b;
                ls[l] = (int8_t)k;
            }
            nc |= nl == 0;
            const int nin = (op == kNot || op == kCopy) ? 1 : ((op == kMux || op == kNMux) ? 3 : 2);
            const int32_t* ins[3] = {in0, in1, in2};
            for (int k = 0; k < 3; k++) idx[k][b] = k < nin ? ins[k][g] : 0;  // unused -> row 0
            idx[3][b] = out[g];
        }
        Plan p = Plan();
        p.count = (int)n;
        p.lanes = (int)lanes;
        p.uniform_op = 0;
        p.ops = (const int8_t*)(dbase + o_ops);
        p.gate_lane0 = (const int32_t*)(dbase + o_l0);
        p.lane_gate = (const int32_t*)(dbase + o_lg);
        p.lane_sub = (const int8_t*)(dbase + o_ls);
        for (int k = 0; k < 3; k++) p.in_idx[k] = (const int32_t*)(dbase + o_idx[k]);
        p.out_idx = (const int32_t*)(dbase + o_idx[3]);
        c->waves.push_back(p);
        c->wave_nc.push_back(nc ? 1 : 0);
    }
    e = cudaMemcpy(c->dbuf, host.data(), total, cudaMemcpyHostToDevice);
    // workspace for the widest wave
    Workspace& ws = c->exec.ws;
    const size_t cap = max_lanes < 1 ? 1 : (size_t)max_lanes;
    if (e == cudaSuccess) e = cudaMalloc(&ws.lane_in, cap * kTlwe0 * 4);
    if (e == cudaSuccess) {
        if (level == CUFHE_LVL02) {
            e = cudaMalloc(&ws.lane_out2, cap * CUFHE_TLWE2_WORDS * 8);
            ws.lane2_cap = cap;
        } else {
            e = cudaMalloc(&ws.lane_out, cap * kTlwe1 * 4);
        }
        ws.lane_cap = cap;
    }
    if (e == cudaSuccess) {
        const int units = level == CUFHE_LVL1 ? max_lanes : max_gates;
        if (units > 0) e = iks_tc_reserve(level == CUFHE_LVL02 ? ws.iks2 : ws.iks, units,
                                          level == CUFHE_LVL02, 0);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking);
    // the plan upload (a pageable copy may return before its DMA ends) and the
    // zeroing above are on the legacy stream, which the engine's non-blocking
    // streams do not wait for: finish them before the circuit can run
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        circuit_free(c);
        return fail(CUFHE_ERR_NOMEM, "circuit buffers: %s", cudaGetErrorString(e));
    }
    *out_c = c;
    return CUFHE_OK;
}

static int sms_of(int device)
{
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        sms = 148;
    }
    return sms;
}

int cufhe_circuit_create(cufhe_circuit_t* out_c, int level, size_t num_wires, size_t num_gates,
                         const int32_t* gate_ops, const int32_t* in0, const int32_t* in1,
                         const int32_t* in2, const int32_t* out, int device)
{
    if (!out_c) return fail(CUFHE_ERR_ARG, "null circuit handle");
    *out_c = nullptr;
    if (level != CUFHE_LVL0 && level != CUFHE_LVL1 && level != CUFHE_LVL02)
        return fail(CUFHE_ERR_ARG, "bad level %d", level);
    if (device < 0) device = 0;
    if (device >= g_gpu_num) return fail(CUFHE_ERR_ARG, "device %d >= gpu num", device);
    std::vector<int32_t> wave;
    int nwaves = 0;
    const int prc = plan_waves(level, num_wires, num_gates, gate_ops, in0, in1, in2, out,
                               sms_of(device), wave, nwaves);
    if (prc != CUFHE_OK) return prc;
    const DeviceState& D = g_dev[device];
    if (level == CUFHE_LVL02 ? !D.ready2 : !D.ready)
        return fail(CUFHE_ERR_STATE, level == CUFHE_LVL02 ? "cufhe_initialize_lvl02() not called"
                                                         : "cufhe_initialize() not called");
    std::vector<std::vector<int32_t>> members(nwaves);
    for (size_t g = 0; g < num_gates; g++) members[wave[g]].push_back((int32_t)g);
    return build_circuit(out_c, level, num_wires, num_gates, gate_ops, in0, in1, in2, out, device,
                         members);
}

int cufhe_circuit_create_split(cufhe_circuit_t* out_c, int level, size_t num_wires,
                               size_t num_gates, const int32_t* gate_ops, const int32_t* in0,
                               const int32_t* in1, const int32_t* in2, const int32_t* out,
                               int device, int parts)
{
    if (!out_c) return fail(CUFHE_ERR_ARG, "null circuit handle");
    *out_c = nullptr;
    if (parts < 1 || parts > 64) return fail(CUFHE_ERR_ARG, "parts %d outside 1..64", parts);
    if (device < 0) device = 0;
    if (device >= g_gpu_num) return fail(CUFHE_ERR_ARG, "device %d >= gpu num", device);
    std::vector<int32_t> wave;
    int nwaves = 0;
    int rc = plan_waves(level, num_wires, num_gates, gate_ops, in0, in1, in2, out, sms_of(device),
                        wave, nwaves);
    if (rc != CUFHE_OK) return rc;
    std::vector<int32_t> group;
    const int ng = parts == 1 ? 1
                              : split_components(num_wires, num_gates, gate_ops, in0, in1, in2,
                                                 out, parts, group);
    if (ng <= 1)
        return cufhe_circuit_create(out_c, level, num_wires, num_gates, gate_ops, in0, in1, in2,
                                    out, device);
    const DeviceState& D = g_dev[device];
    if (level == CUFHE_LVL02 ? !D.ready2 : !D.ready)
        return fail(CUFHE_ERR_STATE, level == CUFHE_LVL02 ? "cufhe_initialize_lvl02() not called"
                                                         : "cufhe_initialize() not called");
    cufhe_circuit_s* c = new cufhe_circuit_s();
    c->device = device;
    c->level = level;
    c->wires = num_wires;
    c->gates = num_gates;
    c->exec.device = device;
    CK(cudaSetDevice(device));
    for (int k = 0; k < ng && rc == CUFHE_OK; k++) {
        // the group's gates, in circuit order, as a circuit of its own over the
        // same wire table
        std::vector<int32_t> ops_k, i0_k, i1_k, i2_k, out_k;
        for (size_t g = 0; g < num_gates; g++) {
            if (group[g] != k) continue;
            ops_k.push_back(gate_ops[g]);
            i0_k.push_back(in0[g]);
            i1_k.push_back(in1 ? in1[g] : -1);
            i2_k.push_back(in2 ? in2[g] : -1);
            out_k.push_back(out[g]);
        }
        std::vector<int32_t> wave_k;
        int nw_k = 0;
        rc = plan_waves(level, num_wires, ops_k.size(), ops_k.data(), i0_k.data(), i1_k.data(),
                        i2_k.data(), out_k.data(), sms_of(device), wave_k, nw_k);
        if (rc != CUFHE_OK) break;
        std::vector<std::vector<int32_t>> members(nw_k);
        for (size_t g = 0; g < ops_k.size(); g++) members[wave_k[g]].push_back((int32_t)g);
        cufhe_circuit_t sub = nullptr;
        rc = build_circuit(&sub, level, num_wires, ops_k.size(), ops_k.data(), i0_k.data(),
                           i1_k.data(), i2_k.data(), out_k.data(), device, members);
        if (rc != CUFHE_OK) break;
        c->parts.push_back(sub);
        c->max_lanes = std::max(c->max_lanes, sub->max_lanes);
        c->max_gates = std::max(c->max_gates, sub->max_gates);
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e == cudaSuccess) c->part_st.push_back(st);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) c->part_done.push_back(ev);
        if (e != cudaSuccess) rc = fail(CUFHE_ERR_CUDA, "circuit part stream: %s", cudaGetErrorString(e));
    }
    if (rc == CUFHE_OK) {
        const cudaError_t e = cudaEventCreateWithFlags(&c->part_fork, cudaEventDisableTiming);
        if (e != cudaSuccess) rc = fail(CUFHE_ERR_CUDA, "circuit fork event: %s", cudaGetErrorString(e));
    }
    if (rc != CUFHE_OK) {
        circuit_free(c);
        return rc;
    }
    *out_c = c;
    return CUFHE_OK;
}

static size_t circuit_waves(const cufhe_circuit_s* c)
{
    size_t n = c->waves.size();
    for (const cufhe_circuit_s* q : c->parts) n = std::max(n, q->waves.size());
    return n;
}

int cufhe_circuit_info(cufhe_circuit_t c, int* waves, int* max_wave_gates, int* max_wave_lanes)
{
    if (!c) return fail(CUFHE_ERR_ARG, "null circuit");
    if (waves) *waves = (int)circuit_waves(c);
    if (max_wave_gates) *max_wave_gates = c->max_gates;
    if (max_wave_lanes) *max_wave_lanes = c->max_lanes;
    return CUFHE_OK;
}

int cufhe_circuit_wave_sizes(cufhe_circuit_t c, int32_t* gates, int32_t* lanes, size_t cap)
{
    if (!c) return fail(CUFHE_ERR_ARG, "null circuit");
    const size_t n = circuit_waves(c);
    for (size_t w = 0; w < n && w < cap; w++) {
        if (gates) gates[w] = 0;
        if (lanes) lanes[w] = 0;
    }
    // a split circuit: wave w of every group runs at the same time; their sum
    const size_t np = c->parts.empty() ? 1 : c->parts.size();
    for (size_t i = 0; i < np; i++) {
        const cufhe_circuit_s* q = c->parts.empty() ? c : c->parts[i];
        for (size_t w = 0; w < q->waves.size() && w < cap; w++) {
            if (gates) gates[w] += q->waves[w].count;
            if (lanes) lanes[w] += q->waves[w].lanes;
        }
    }
    return (int)n;
}

// Runs circuit c (or each group of a split circuit, on the group's own
// stream, forked from and joined back into st) over `wires` on stream st.
static int circuit_run_on(cufhe_circuit_s* c, uint32_t* wires, cudaStream_t st, bool graph)
{
    if (!c->parts.empty()) {
        CK(cudaEventRecord(c->part_fork, st));
        for (size_t i = 0; i < c->parts.size(); i++) {
            CK(cudaStreamWaitEvent(c->part_st[i], c->part_fork, 0));
            const int rc = circuit_run_on(c->parts[i], wires, c->part_st[i], graph);
            // joined even when the group failed part-way, so that the caller's
            // stream still orders after whatever the group did launch
            CK(cudaEventRecord(c->part_done[i], c->part_st[i]));
            CK(cudaStreamWaitEvent(st, c->part_done[i], 0));
            if (rc) return rc;
        }
        return CUFHE_OK;
    }
    if (!graph) {
        c->exec.st = st;
        for (size_t w = 0; w < c->waves.size(); w++) {
            const int rc = run_wave(c, w, wires);
            if (rc) return rc;
        }
        return CUFHE_OK;
    }
    if (!c->gexec || c->graph_wires != wires || c->graph_precision != g_precision) {
        const int rc = circuit_capture(c, wires, st);
        if (rc) return rc;
    }
    CK(cudaGraphLaunch(c->gexec, st));
    g_launches.fetch_add(c->graph_launches);
    return CUFHE_OK;
}

int cufhe_circuit_run(cufhe_circuit_t c, uint32_t* wires, cufhe_stream_t st, int use_graph)
{
    if (!c || !wires) return fail(CUFHE_ERR_ARG, "null circuit or wire table");
    cufhe_stream_s* s = resolve(st);
    if (s->device != c->device)
        return fail(CUFHE_ERR_ARG, "circuit lives on device %d, stream on %d", c->device, s->device);
    const DeviceState& D = g_dev[c->device];
    if (c->level == CUFHE_LVL02 ? !D.ready2 : !D.ready)
        return fail(CUFHE_ERR_STATE, "keys of the circuit's level are not initialised");
    CK(cudaSetDevice(c->device));
    return circuit_run_on(c, wires, s->st, use_graph != 0);
}

int cufhe_circuit_destroy(cufhe_circuit_t c)
{
    if (!c) return CUFHE_OK;
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    circuit_free(c);
    return CUFHE_OK;
}

// ---- sharding over devices --------------------------------------------------
// The reference spreads gates over GPUs by giving each Stream a device in
// turn, with every key replicated per device (include/cufhe_gpu.cuh:164-175,
// src/cufhe_gates_gpu.cu:38-61).  Here one batch or one circuit is split over
// `shards` shards, shard s running on device s % cufhe_set_gpu_num.  A batch
// splits into contiguous gate ranges of balanced blind-rotation lanes; a
// circuit splits every wave, and the wires one shard writes and another reads
// later are copied into the reader's own wire table right after the wave
// that writes them (stores from the writer's device into the peer's memory
// over NVLink; no multicast).  The planners are host functions and need no
// GPU.

namespace cufhe {
namespace {

constexpr int kMaxShards = 64;

static int ninputs(int op) { return (op == kNot || op == kCopy) ? 1 : ((op == kMux || op == kNMux) ? 3 : 2); }

// Contiguous gate ranges [bounds[k], bounds[k + 1]) with balanced lanes (by
// count when no gate bootstraps).
static void plan_batch_shards(const int32_t* gates, int uniform, size_t count, int shards,
                              std::vector<size_t>& bounds)
{
    bounds.assign((size_t)shards + 1, count);
    bounds[0] = 0;
    size_t total = 0;
    for (size_t b = 0; b < count; b++) total += lanes_of_gate(gates ? gates[b] : uniform);
    if (total == 0) {
        for (int k = 1; k < shards; k++) bounds[k] = count * (size_t)k / (size_t)shards;
        return;
    }
    size_t acc = 0;
    int k = 1;
    for (size_t b = 0; b < count && k < shards; b++) {
        acc += lanes_of_gate(gates ? gates[b] : uniform);
        while (k < shards && acc * (size_t)shards >= total * (size_t)k) bounds[k++] = b + 1;
    }
}

// Waves (plan_waves) and a shard per gate: within a wave the lanes are
// balanced (at most ceil(lanes / shards) per shard unless a gate does not
// fit anywhere else), and a gate goes to the shard that wrote most of its
// operands when that shard has room, which keeps chains of gates on one
// shard and the copies few.  copies = wires that must move between shards.
static int plan_shards(int level, size_t num_wires, size_t num_gates, const int32_t* gate_ops,
                       const int32_t* in0, const int32_t* in1, const int32_t* in2,
                       const int32_t* out, int sms, int shards, std::vector<int32_t>& wave,
                       int& nwaves, std::vector<int32_t>& shard, std::vector<uint64_t>& copies)
{
    if (shards < 1 || shards > kMaxShards)
        return fail(CUFHE_ERR_ARG, "shards %d outside [1, %d]", shards, kMaxShards);
    const int rc = plan_waves(level, num_wires, num_gates, gate_ops, in0, in1, in2, out, sms, wave,
                              nwaves);
    if (rc != CUFHE_OK) return rc;
    std::vector<int32_t> producer(num_wires, -1);
    for (size_t g = 0; g < num_gates; g++) producer[out[g]] = (int32_t)g;
    std::vector<std::vector<int32_t>> members(nwaves);
    for (size_t g = 0; g < num_gates; g++) members[wave[g]].push_back((int32_t)g);
    shard.assign(num_gates, 0);
    const int32_t* ins[3] = {in0, in1, in2};
    for (int w = 0; w < nwaves; w++) {
        long lanes = 0;
        for (int32_t g : members[w]) lanes += lanes_of_gate(gate_ops[g]);
        const long target = (lanes + shards - 1) / shards;
        std::vector<long> load(shards, 0), light(shards, 0);
        for (int32_t g : members[w]) {
            const int op = gate_ops[g];
            int votes[3] = {-1, -1, -1}, pref = -1, best = 0;
            for (int k = 0; k < ninputs(op); k++) {
                const int32_t pg = producer[ins[k][g]];
                votes[k] = pg >= 0 ? shard[pg] : -1;
            }
            for (int k = 0; k < 3; k++) {
                if (votes[k] < 0) continue;
                int n = 0;
                for (int q = 0; q < 3; q++) n += votes[q] == votes[k];
                if (n > best) best = n, pref = votes[k];
            }
            const long lg = lanes_of_gate(op);
            int sh;
            if (lg == 0) {  // Not / Copy: no rotation, stay with the operand
                sh = pref;
                if (sh < 0) {
                    sh = 0;
                    for (int q = 1; q < shards; q++) sh = light[q] < light[sh] ? q : sh;
                }
                light[sh]++;
            } else if (pref >= 0 && load[pref] + lg <= target) {
                sh = pref;
            } else {
                sh = 0;
                for (int q = 1; q < shards; q++) sh = load[q] < load[sh] ? q : sh;
            }
            load[sh] += lg;
            shard[g] = sh;
        }
    }
    // wires to move: (wave of the writer, writer shard, reader shard, wire)
    copies.clear();
    for (size_t g = 0; g < num_gates; g++)
        for (int k = 0; k < ninputs(gate_ops[g]); k++) {
            const int32_t x = ins[k][g], pg = producer[x];
            if (pg < 0 || shard[pg] == shard[g]) continue;
            copies.push_back(((uint64_t)wave[pg] << 44) | ((uint64_t)shard[pg] << 38) |
                             ((uint64_t)shard[g] << 32) | (uint32_t)x);
        }
    std::sort(copies.begin(), copies.end());
    copies.erase(std::unique(copies.begin(), copies.end()), copies.end());
    return CUFHE_OK;
}

}  // namespace
}  // namespace cufhe

// A circuit split over shards: one sub-circuit per shard (its gates of every
// wave; waves may be empty) and, per wave, the wires each shard sends to
// each other shard.
struct cufhe_sharded_s {
    int level = 0, shards = 0, nwaves = 0, words = 0;
    size_t wires = 0, ncopies = 0;
    std::vector<cufhe_circuit_s*> sub;
    std::vector<int> device;
    struct Copy {
        int wave, from, to;
        const int32_t* rows;  // on the sending shard's device
        int n;
    };
    std::vector<Copy> copies;       // ordered by wave
    std::vector<const int32_t*> outs;  // every wire a shard's gates write
    std::vector<int> nouts;
    std::vector<void*> rowbuf;
    std::vector<cudaStream_t> st;
    std::vector<cudaEvent_t> ev;
};

namespace cufhe {
namespace {

void sharded_free(cufhe_sharded_s* c)
{
    for (size_t s = 0; s < c->sub.size(); s++) {
        cudaSetDevice(c->device[s]);
        if (s < c->st.size() && c->st[s]) cudaStreamSynchronize(c->st[s]);
        if (c->sub[s]) circuit_free(c->sub[s]);
        if (s < c->rowbuf.size() && c->rowbuf[s]) cudaFree(c->rowbuf[s]);
        if (s < c->ev.size() && c->ev[s]) cudaEventDestroy(c->ev[s]);
        if (s < c->st.size() && c->st[s]) cudaStreamDestroy(c->st[s]);
    }
    delete c;
}

}  // namespace
}  // namespace cufhe

using namespace cufhe;

int cufhe_batch_shard_plan(const int32_t* gates_host, int uniform_gate, size_t count, int shards,
                           size_t* bounds)
{
    if (!bounds) return fail(CUFHE_ERR_ARG, "null bounds");
    if (shards < 1 || shards > kMaxShards)
        return fail(CUFHE_ERR_ARG, "shards %d outside [1, %d]", shards, kMaxShards);
    std::vector<size_t> b;
    plan_batch_shards(gates_host, uniform_gate, count, shards, b);
    for (int k = 0; k <= shards; k++) bounds[k] = b[k];
    return CUFHE_OK;
}

int cufhe_gate_batch_sharded_host(const int32_t* gates_host, int uniform_gate, size_t count,
                                  int level, uint32_t* out_host, const uint32_t* in0_host,
                                  const uint32_t* in1_host, const uint32_t* in2_host, int shards)
{
    if (shards <= 0) shards = g_gpu_num;
    if (shards > kMaxShards) return fail(CUFHE_ERR_ARG, "shards %d > %d", shards, kMaxShards);
    if (level != CUFHE_LVL0 && level != CUFHE_LVL1 && level != CUFHE_LVL02)
        return fail(CUFHE_ERR_ARG, "bad level %d", level);
    if (count == 0) return CUFHE_OK;
    if (!out_host || !in0_host) return fail(CUFHE_ERR_ARG, "null ciphertext pointer");
    const size_t words = level == CUFHE_LVL1 ? kTlwe1 : kTlwe0;
    std::vector<size_t> bounds;
    plan_batch_shards(gates_host, uniform_gate, count, shards, bounds);
    // one engine stream per shard, on device shard % gpu num
    for (int k = 0; k < shards; k++) {
        const int dev = k % g_gpu_num;
        if (k < (int)g_shard_st.size() && g_shard_st[k]->device != dev) {
            cufhe_stream_destroy(g_shard_st[k]);
            g_shard_st[k] = nullptr;
        }
        if (k >= (int)g_shard_st.size()) g_shard_st.push_back(nullptr);
        if (!g_shard_st[k]) {
            const int rc = cufhe_stream_create(&g_shard_st[k], dev);
            if (rc) return rc;
        }
    }
    for (int k = 0; k < shards; k++) {
        const size_t b0 = bounds[k], n = bounds[k + 1] - b0;
        if (!n) continue;
        const int rc = cufhe_gate_batch_host(
            gates_host ? gates_host + b0 : nullptr, uniform_gate, n, level, out_host + b0 * words,
            in0_host + b0 * words, in1_host ? in1_host + b0 * words : nullptr,
            in2_host ? in2_host + b0 * words : nullptr, g_shard_st[k]);
        if (rc) return rc;
    }
    for (int k = 0; k < shards; k++) {
        const int rc = cufhe_stream_synchronize(g_shard_st[k]);
        if (rc) return rc;
    }
    return CUFHE_OK;
}

int cufhe_circuit_shard_plan(int level, size_t num_wires, size_t num_gates, const int32_t* gate_ops,
                             const int32_t* in0, const int32_t* in1, const int32_t* in2,
                             const int32_t* out, int sms, int shards, int32_t* wave_of_gate,
                             int32_t* shard_of_gate, int* num_waves, size_t* num_copies)
{
    if (!wave_of_gate || !shard_of_gate || !num_waves) return fail(CUFHE_ERR_ARG, "null plan output");
    std::vector<int32_t> wave, shard;
    std::vector<uint64_t> copies;
    int nwaves = 0;
    const int rc = plan_shards(level, num_wires, num_gates, gate_ops, in0, in1, in2, out, sms,
                               shards, wave, nwaves, shard, copies);
    if (rc != CUFHE_OK) return rc;
    for (size_t g = 0; g < num_gates; g++) {
        wave_of_gate[g] = wave[g];
        shard_of_gate[g] = shard[g];
    }
    *num_waves = nwaves;
    if (num_copies) *num_copies = copies.size();
    return CUFHE_OK;
}

int cufhe_sharded_create(cufhe_sharded_t* out_c, int level, size_t num_wires, size_t num_gates,
                         const int32_t* gate_ops, const int32_t* in0, const int32_t* in1,
                         const int32_t* in2, const int32_t* out, int shards)
{
    if (!out_c) return fail(CUFHE_ERR_ARG, "null circuit handle");
    *out_c = nullptr;
    if (shards <= 0) shards = g_gpu_num;
    std::vector<int32_t> wave, shard;
    std::vector<uint64_t> copies;
    int nwaves = 0;
    int rc = plan_shards(level, num_wires, num_gates, gate_ops, in0, in1, in2, out, sms_of(0),
                         shards, wave, nwaves, shard, copies);
    if (rc != CUFHE_OK) return rc;
    for (int k = 0; k < shards && k < g_gpu_num; k++) {
        const DeviceState& D = g_dev[k];
        if (level == CUFHE_LVL02 ? !D.ready2 : !D.ready)
            return fail(CUFHE_ERR_STATE, "keys of the circuit's level are not initialised on "
                                         "device %d", k);
    }
    cufhe_sharded_s* c = new cufhe_sharded_s();
    c->level = level;
    c->shards = shards;
    c->nwaves = nwaves;
    c->wires = num_wires;
    c->words = level == CUFHE_LVL1 ? kTlwe1 : kTlwe0;
    c->ncopies = copies.size();
    c->sub.assign(shards, nullptr);
    c->rowbuf.assign(shards, nullptr);
    c->st.assign(shards, nullptr);
    c->ev.assign(shards, nullptr);
    c->outs.assign(shards, nullptr);
    c->nouts.assign(shards, 0);
    for (int k = 0; k < shards; k++) c->device.push_back(k % g_gpu_num);
    // peer access between the devices in use (stores into a peer's table)
    for (int a = 0; a < shards && a < g_gpu_num; a++)
        for (int b = 0; b < shards && b < g_gpu_num; b++) {
            if (a == b) continue;
            int ok = 0;
            cudaDeviceCanAccessPeer(&ok, a, b);
            if (!ok) {
                sharded_free(c);
                return fail(CUFHE_ERR_STATE, "device %d cannot access device %d's memory", a, b);
            }
            cudaSetDevice(a);
            const cudaError_t e = cudaDeviceEnablePeerAccess(b, 0);
            if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled) {
                sharded_free(c);
                return fail(CUFHE_ERR_CUDA, "peer access %d -> %d: %s", a, b, cudaGetErrorString(e));
            }
            cudaGetLastError();
        }
    // per shard: the sub-circuit, and one device buffer with its outgoing
    // copy rows (grouped by wave and reader) followed by its output rows
    for (int k = 0; k < shards; k++) {
        std::vector<std::vector<int32_t>> members(nwaves);
        std::vector<int32_t> rows;
        for (size_t g = 0; g < num_gates; g++)
            if (shard[g] == k) members[wave[g]].push_back((int32_t)g);
        rc = build_circuit(&c->sub[k], level, num_wires, num_gates, gate_ops, in0, in1, in2, out,
                           c->device[k], members);
        if (rc != CUFHE_OK) {
            sharded_free(c);
            return rc;
        }
        struct Pending { int wave, to; size_t off; int n; };
        std::vector<Pending> mine;
        for (size_t i = 0; i < copies.size();) {
            const uint64_t key = copies[i] >> 32;
            const int w = (int)(key >> 12), from = (int)((key >> 6) & 63), to = (int)(key & 63);
            size_t j = i;
            while (j < copies.size() && (copies[j] >> 32) == key) j++;
            if (from == k) {
                mine.push_back({w, to, rows.size(), (int)(j - i)});
                for (size_t q = i; q < j; q++) rows.push_back((int32_t)(copies[q] & 0xFFFFFFFFu));
            }
            i = j;
        }
        const size_t out_off = rows.size();
        for (size_t g = 0; g < num_gates; g++)
            if (shard[g] == k) rows.push_back(out[g]);
        cudaError_t e = cudaSetDevice(c->device[k]);
        if (e == cudaSuccess && !rows.empty()) e = cudaMalloc(&c->rowbuf[k], rows.size() * 4);
        if (e == cudaSuccess && !rows.empty())
            e = cudaMemcpy(c->rowbuf[k], rows.data(), rows.size() * 4, cudaMemcpyHostToDevice);
        // a pageable copy may return before its DMA ends, and the shard streams
        // are non-blocking: finish it before they can read the rows
        if (e == cudaSuccess && !rows.empty()) e = cudaStreamSynchronize(0);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st[k], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev[k], cudaEventDisableTiming);
        if (e != cudaSuccess) {
            sharded_free(c);
            return fail(CUFHE_ERR_NOMEM, "sharded circuit buffers: %s", cudaGetErrorString(e));
        }
        const int32_t* base = static_cast<const int32_t*>(c->rowbuf[k]);
        for (const Pending& q : mine) c->copies.push_back({q.wave, k, q.to, base + q.off, q.n});
        c->outs[k] = base + out_off;
        c->nouts[k] = (int)(rows.size() - out_off);
    }
    std::stable_sort(c->copies.begin(), c->copies.end(),
                     [](const cufhe_sharded_s::Copy& a, const cufhe_sharded_s::Copy& b) {
                         return a.wave < b.wave;
                     });
    *out_c = c;
    return CUFHE_OK;
}

int cufhe_sharded_info(cufhe_sharded_t c, int* waves, size_t* copies, int* shards)
{
    if (!c) return fail(CUFHE_ERR_ARG, "null circuit");
    if (waves) *waves = c->nwaves;
    if (copies) *copies = c->ncopies;
    if (shards) *shards = c->shards;
    return CUFHE_OK;
}

int cufhe_sharded_device(cufhe_sharded_t c, int shard)
{
    if (!c || shard < 0 || shard >= c->shards) return fail(CUFHE_ERR_ARG, "bad shard");
    return c->device[shard];
}

int cufhe_sharded_run(cufhe_sharded_t c, uint32_t* const* wires)
{
    if (!c || !wires) return fail(CUFHE_ERR_ARG, "null circuit or wire tables");
    for (int k = 0; k < c->shards; k++)
        if (!wires[k]) return fail(CUFHE_ERR_ARG, "null wire table of shard %d", k);
    for (int k = 0; k < c->shards && k < g_gpu_num; k++)
        if (c->level == CUFHE_LVL02 ? !g_dev[k].ready2 : !g_dev[k].ready)
            return fail(CUFHE_ERR_STATE, "keys of the circuit's level are not initialised");
    size_t ci = 0;
    std::vector<char> sent(c->shards);
    for (int w = 0; w < c->nwaves; w++) {
        for (int k = 0; k < c->shards; k++) {
            CK(cudaSetDevice(c->device[k]));
            c->sub[k]->exec.st = c->st[k];
            const int rc = run_wave(c->sub[k], w, wires[k]);
            if (rc) return rc;
        }
        // this wave's copies, on the writer's stream right after its gates;
        // each reader waits for its writers before its next wave
        const size_t c0 = ci;
        std::fill(sent.begin(), sent.end(), 0);
        for (; ci < c->copies.size() && c->copies[ci].wave == w; ci++) {
            const cufhe_sharded_s::Copy& q = c->copies[ci];
            CK(cudaSetDevice(c->device[q.from]));
            LAUNCH(CUFHE_K_FINALIZE, c->st[q.from],
                   launch_copy_rows(q.rows, q.n, c->words, wires[q.from], wires[q.to],
                                    c->st[q.from]));
            sent[q.from] = 1;
        }
        for (int k = 0; k < c->shards; k++)
            if (sent[k]) {
                CK(cudaSetDevice(c->device[k]));
                CK(cudaEventRecord(c->ev[k], c->st[k]));
            }
        for (size_t q = c0; q < ci; q++) {
            const cufhe_sharded_s::Copy& cp = c->copies[q];
            CK(cudaSetDevice(c->device[cp.to]));
            CK(cudaStreamWaitEvent(c->st[cp.to], c->ev[cp.from], 0));
        }
    }
    return CUFHE_OK;
}

int cufhe_sharded_collect(cufhe_sharded_t c, uint32_t* const* wires, int dst)
{
    if (!c || !wires) return fail(CUFHE_ERR_ARG, "null circuit or wire tables");
    if (dst < 0 || dst >= c->shards) return fail(CUFHE_ERR_ARG, "bad shard %d", dst);
    for (int k = 0; k < c->shards; k++) {
        if (k == dst || !c->nouts[k]) continue;
        CK(cudaSetDevice(c->device[k]));
        LAUNCH(CUFHE_K_FINALIZE, c->st[k],
               launch_copy_rows(c->outs[k], c->nouts[k], c->words, wires[k], wires[dst], c->st[k]));
        CK(cudaEventRecord(c->ev[k], c->st[k]));
        CK(cudaSetDevice(c->device[dst]));
        CK(cudaStreamWaitEvent(c->st[dst], c->ev[k], 0));
    }
    return CUFHE_OK;
}

int cufhe_sharded_synchronize(cufhe_sharded_t c)
{
    if (!c) return fail(CUFHE_ERR_ARG, "null circuit");
    for (int k = 0; k < c->shards; k++) {
        CK(cudaSetDevice(c->device[k]));
        CK(cudaStreamSynchronize(c->st[k]));
    }
    return cufhe_synchronize();
}

int cufhe_sharded_destroy(cufhe_sharded_t c)
{
    if (!c) return CUFHE_OK;
    sharded_free(c);
    return CUFHE_OK;
}

int cufhe_initialize_cb(const cufhe_cbkeyview* kv)
{
    if (!kv || !kv->privks0 || !kv->privks1) return fail(CUFHE_ERR_ARG, "null key view");
    const uint64_t want = (uint64_t)(CUFHE_LVL2_N + 1) * 10 * 15 * CUFHE_TRLWE1_WORDS;
    if (kv->words != want)
        return fail(CUFHE_ERR_ARG, "private key-switching key has %zu words, expected %llu",
                    kv->words, (unsigned long long)want);
    int avail = 0;
    if (cudaGetDeviceCount(&avail) != cudaSuccess || avail == 0)
        return fail(CUFHE_ERR_CUDA, "no CUDA device visible");
    for (int d = 0; d < g_gpu_num; d++) {
        if (g_dev[d].ready_cb) release_cb(d);
        const int rc = init_cb(d, kv);
        if (rc) {
            release_cb(d);
            return rc;
        }
    }
    cudaSetDevice(0);
    return CUFHE_OK;
}

int cufhe_cleanup_cb(void)
{
    for (int d = 0; d < kMaxDev; d++)
        if (g_dev[d].ready_cb) release_cb(d);
    cudaSetDevice(0);
    return CUFHE_OK;
}

int cufhe_private_keyswitch(const uint64_t* tlwe2, size_t count, int func, uint32_t* trlwe_out,
                            cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    const DeviceState& D = g_dev[s->device];
    if (!D.ready_cb) return fail(CUFHE_ERR_STATE, "cufhe_initialize_cb() not called");
    if (!tlwe2 || !trlwe_out) return fail(CUFHE_ERR_ARG, "null pointer");
    if (func != 0 && func != 1) return fail(CUFHE_ERR_ARG, "bad key-switching function %d", func);
    if (count == 0) return CUFHE_OK;
    if (count > (1u << 24)) return fail(CUFHE_ERR_ARG, "too many inputs");
    CK(cudaSetDevice(s->device));
    PksMap map = {};
    map.per = (int)count;
    map.stride_lo = CUFHE_TRLWE1_WORDS;
    return run_privks(s, tlwe2, (int)count, func, map, trlwe_out);
}

int cufhe_circuit_bootstrap(const uint32_t* tlwe0, size_t count, uint32_t* trgsw_out,
                            cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    const DeviceState& D = g_dev[s->device];
    if (!D.ready_cb) return fail(CUFHE_ERR_STATE, "cufhe_initialize_cb() not called");
    if (!D.ready2) return fail(CUFHE_ERR_STATE, "cufhe_initialize_lvl02() not called");
    if (!tlwe0 || !trgsw_out) return fail(CUFHE_ERR_ARG, "null pointer");
    if (count == 0) return CUFHE_OK;
    if (count > (1u << 22)) return fail(CUFHE_ERR_ARG, "too many inputs");
    CK(cudaSetDevice(s->device));
    int rc = ensure_lane2(s, 3 * count);
    if (rc) return rc;
    uint64_t* t2 = s->ws.lane_out2;
    constexpr int kL = 3, kBgbit = 6;
    PksMap map = {};
    map.per = (int)count;  // unit u = i * count + bit
    map.stride_lo = (size_t)2 * kL * CUFHE_TRLWE1_WORDS;
    map.stride_hi = CUFHE_TRLWE1_WORDS;
    for (int i = 0; i < kL; i++) map.badd[i] = 1ull << (64 - (i + 1) * kBgbit - 1);
    if (g_precision == CUFHE_INT8_EXACT) {
        for (int i = 0; i < kL; i++) {
            rc = run_br2(s, tlwe0, (int)count, map.badd[i], -1, nullptr,
                         t2 + (size_t)i * count * CUFHE_TLWE2_WORDS);
            if (rc) return rc;
        }
    } else {
        // one launch for the three digits: lane i count + b rotates bit b with
        // test value mu_0 >> 6 i = mu_i (fills the partial last wave of each)
        rc = run_br2(s, tlwe0, (int)(kL * count), map.badd[0], -1, nullptr, t2, (int)count, kBgbit);
        if (rc) return rc;
    }
    for (int f = 0; f < 2; f++) {
        rc = run_privks(s, t2, (int)(3 * count), f, map,
                        trgsw_out + (size_t)f * kL * CUFHE_TRLWE1_WORDS, f == 0);
        if (rc) return rc;
    }
    return CUFHE_OK;
}

static int gadget_rows(int gadget) { return gadget == CUFHE_GADGET_CB ? 6 : 4; }

int cufhe_trgsw_to_fft(int gadget, const uint32_t* trgsw, size_t count, double* fft_out,
                       cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    const DeviceState& D = g_dev[s->device];
    if (gadget != CUFHE_GADGET_LVL1 && gadget != CUFHE_GADGET_CB)
        return fail(CUFHE_ERR_ARG, "bad gadget %d", gadget);
    if (!trgsw || !fft_out) return fail(CUFHE_ERR_ARG, "null pointer");
    const double2* psi = D.ready_cb ? D.cb_psi : D.psi;
    const double2* tw = D.ready_cb ? D.cb_tw512 : D.tw512;
    if (!psi) return fail(CUFHE_ERR_STATE, "cufhe_initialize() or cufhe_initialize_cb() not called");
    if (count == 0) return CUFHE_OK;
    if (count > (1u << 22)) return fail(CUFHE_ERR_ARG, "too many TRGSWs");
    CK(cudaSetDevice(s->device));
    const Fp64Tables t = {psi, tw};
    LAUNCH(CUFHE_K_CMUX, s->st,
           launch_bk_to_fft(trgsw, (int)(count * 2 * gadget_rows(gadget)), t,
                            reinterpret_cast<double2*>(fft_out), s->st));
    return CUFHE_OK;
}

int cufhe_cmux(int gadget, const double* trgsw_fft, const uint32_t* d1, const uint32_t* d0,
               uint32_t* out, size_t count, cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    const DeviceState& D = g_dev[s->device];
    if (gadget != CUFHE_GADGET_LVL1 && gadget != CUFHE_GADGET_CB)
        return fail(CUFHE_ERR_ARG, "bad gadget %d", gadget);
    if (!trgsw_fft || !d1 || !d0 || !out) return fail(CUFHE_ERR_ARG, "null pointer");
    const double2* psi = D.ready_cb ? D.cb_psi : D.psi;
    const double2* tw = D.ready_cb ? D.cb_tw512 : D.tw512;
    if (!psi) return fail(CUFHE_ERR_STATE, "cufhe_initialize() or cufhe_initialize_cb() not called");
    if (count == 0) return CUFHE_OK;
    if (count > (1u << 24)) return fail(CUFHE_ERR_ARG, "too many CMUXes");
    CK(cudaSetDevice(s->device));
    CmuxPlan p = {};
    p.count = (int)count;
    p.per = 1;
    p.node_stride_g = 1;
    p.d0 = d0;
    p.d1 = d1;
    p.trgsw = reinterpret_cast<const double2*>(trgsw_fft);
    p.trgsw_stride = (size_t)2 * gadget_rows(gadget) * 512;
    p.out = out;
    const Fp64Tables t = {psi, tw};
    LAUNCH(CUFHE_K_CMUX, s->st, launch_cmux(gadget, p, t, s->st));
    return CUFHE_OK;
}

int cufhe_lut_eval(const uint8_t* luts_host, size_t num_luts, const double* trgsw_fft,
                   uint32_t mu, uint32_t* tlwe1_out, cufhe_stream_t st)
{
    cufhe_stream_s* s = resolve(st);
    const DeviceState& D = g_dev[s->device];
    if (!luts_host || !trgsw_fft || !tlwe1_out) return fail(CUFHE_ERR_ARG, "null pointer");
    const double2* psi = D.ready_cb ? D.cb_psi : D.psi;
    const double2* tw = D.ready_cb ? D.cb_tw512 : D.tw512;
    if (!psi) return fail(CUFHE_ERR_STATE, "cufhe_initialize() or cufhe_initialize_cb() not called");
    if (num_luts == 0) return CUFHE_OK;
    if (num_luts > (1u << 16)) return fail(CUFHE_ERR_ARG, "too many lookup tables");
    CK(cudaSetDevice(s->device));
    Workspace& w = s->ws;
    const int q = (int)num_luts;
    if (num_luts > w.lut_cap) {
        CK(cudaStreamSynchronize(s->st));
        cudaFree(w.lut_a);
        cudaFree(w.lut_b);
        cudaFree(w.lut_tab);
        w.lut_a = w.lut_b = nullptr;
        w.lut_tab = nullptr;
        w.lut_cap = 0;
        if (cudaMalloc(&w.lut_a, num_luts * 256 * kTrlwe * 4) != cudaSuccess ||
            cudaMalloc(&w.lut_b, num_luts * 128 * kTrlwe * 4) != cudaSuccess ||
            cudaMalloc(&w.lut_tab, num_luts * 256) != cudaSuccess)
            return fail(CUFHE_ERR_NOMEM, "lookup-table buffers for %zu tables", num_luts);
        w.lut_cap = num_luts;
    }
    CK(cudaMemcpyAsync(w.lut_tab, luts_host, num_luts * 256, cudaMemcpyHostToDevice, s->st));
    LAUNCH(CUFHE_K_CMUX, s->st, launch_lut_leaves(w.lut_tab, q, mu, w.lut_a, s->st));
    const Fp64Tables t = {psi, tw};
    const size_t trgsw_words = (size_t)2 * gadget_rows(CUFHE_GADGET_CB) * 512;  // double2
    uint32_t* in = w.lut_a;
    uint32_t* outb = w.lut_b;
    for (int k = 0, width = 128; k < 8; k++, width >>= 1) {
        CmuxPlan p = {};
        p.per = width;  // CMUXes per table at this level
        p.count = q * width;
        p.node_stride_g = (size_t)2 * width;
        p.node_stride_m = 2;
        p.d0 = in;
        p.d1 = in + kTrlwe;
        p.trgsw = reinterpret_cast<const double2*>(trgsw_fft) + (size_t)k * trgsw_words;
        p.trgsw_stride = 8 * trgsw_words;
        p.out = outb;
        LAUNCH(CUFHE_K_CMUX, s->st, launch_cmux(CUFHE_GADGET_CB, p, t, s->st));
        uint32_t* tmp = in;
        in = outb;
        outb = tmp;
    }
    LAUNCH(CUFHE_K_CMUX, s->st, launch_extract8(in, q, tlwe1_out, s->st));
    return CUFHE_OK;
}

int cufhe_autotune(void)
{
    int d = 0;
    CK(cudaGetDevice(&d));
    return autotune_br(d);
}

int cufhe_autotune_table(int32_t* lanes, int32_t* lanes_per_cta, int cap)
{
    int d = 0;
    CK(cudaGetDevice(&d));
    int b[32], g[32];
    const int n = br_fp64_get_tuning(d, b, g, 32);
    for (int i = 0; i < n && i < cap; i++) {
        if (lanes) lanes[i] = b[i];
        if (lanes_per_cta) lanes_per_cta[i] = g[i];
    }
    return n;
}

int cufhe_profile_enable(int on)
{
    g_prof = on != 0;
    return CUFHE_OK;
}

int cufhe_profile_reset(void)
{
    for (auto& r : g_prof_recs) {
        cudaEventSynchronize(r.b);
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    g_prof_recs.clear();
    for (int i = 0; i < CUFHE_K_CLASSES; i++) {
        g_prof_ms[i] = 0;
        g_prof_n[i] = 0;
    }
    return CUFHE_OK;
}

int cufhe_profile_read(int cls, double* total_ms, uint64_t* launches)
{
    if (cls < 0 || cls >= CUFHE_K_CLASSES || !total_ms || !launches)
        return fail(CUFHE_ERR_ARG, "bad profile query");
    for (auto& r : g_prof_recs) {
        CK(cudaEventSynchronize(r.b));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, r.a, r.b));
        g_prof_ms[r.cls] += ms;
        g_prof_n[r.cls] += 1;
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    g_prof_recs.clear();
    *total_ms = g_prof_ms[cls];
    *launches = g_prof_n[cls];
    return CUFHE_OK;
}

const char* cufhe_last_error(void) { return g_err; }

uint64_t cufhe_kernel_launches(void) { return g_launches.load(); }

int cufhe_device_ok(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return 0;
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, 0) != cudaSuccess) return 0;
    return p.major == 10 ? 1 : 0;
}

}  // extern "C"
