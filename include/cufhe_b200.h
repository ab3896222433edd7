/*
 * cufhe_b200.h -- C-ABI of the B200 TFHE gate-bootstrapping engine.
 *
 * Drop-in boundary for cuFHEpp's gate API (include/cufhe_gpu.cuh:42-358 and
 * src/cufhe_gates_gpu.cu:34-824).  The reference exposes C++ templates over
 * TFHEpp types; this header exposes the same operations as plain C functions
 * over pointers and sizes.  include/cufhe_gpu.hpp rebuilds the reference's
 * C++ names (cufhe::Initialize, cufhe::Nand<P>, cufhe::Stream, ...) on top.
 *
 * Conventions
 *  - Every function returns CUFHE_OK (0) or a negative CUFHE_ERR_* code; the
 *    reference prints and exit(-1)s instead (include/error_gpu.cuh:30-66).
 *    cufhe_last_error() describes the most recent failure.
 *  - Ciphertexts use TFHEpp layouts: TLWE<lvl0> = uint32_t[637],
 *    TLWE<lvl1> = uint32_t[1025], b last.
 *  - Gate calls are asynchronous on the given stream; results are valid after
 *    cufhe_synchronize() or once cufhe_stream_query() returns 1, as in the
 *    reference (include/cufhe_gpu.cuh:70-76, src/cufhe_gates_gpu.cu:104-114).
 *  - Not thread-safe, like the reference (global key state).
 */
#ifndef CUFHE_B200_H
#define CUFHE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define CUFHE_OK 0
#define CUFHE_ERR_ARG (-1)         /* bad argument (size, pointer, id) */
#define CUFHE_ERR_STATE (-2)       /* not initialized / wrong key form */
#define CUFHE_ERR_CUDA (-3)        /* CUDA runtime error */
#define CUFHE_ERR_NOMEM (-4)       /* device or host allocation failed */
#define CUFHE_ERR_UNSUPPORTED (-5) /* feature not available in this build */

/* ---- gate ids (the 14 gates of include/cufhe_gpu.cuh:230-358) -------- */
#define CUFHE_NAND 0
#define CUFHE_OR 1
#define CUFHE_ORYN 2
#define CUFHE_ORNY 3
#define CUFHE_AND 4
#define CUFHE_ANDYN 5
#define CUFHE_ANDNY 6
#define CUFHE_NOR 7
#define CUFHE_XOR 8
#define CUFHE_XNOR 9
#define CUFHE_NOT 10
#define CUFHE_COPY 11
#define CUFHE_MUX 12  /* out = in0 ? in1 : in2   (Mux(out, inc, in1, in0)) */
#define CUFHE_NMUX 13 /* out = !(in0 ? in1 : in2) */

/* ---- ciphertext level of a gate call -------------------------------- */
/* CUFHE_LVL0: Ctxt<lvl0param> I/O, blind rotation then key switching
 *             (src/cufhe_gates_gpu.cu:198-511)
 * CUFHE_LVL1: Ctxt<lvl1param> I/O, key switching then blind rotation
 *             (src/cufhe_gates_gpu.cu:513-824) */
#define CUFHE_LVL0 0
#define CUFHE_LVL1 1
/* CUFHE_LVL02: Ctxt<lvl0param> I/O through lvl02 bootstrapping: blind
 *              rotation to lvl2 (N = 2048, Torus64), then key switching
 *              lvl2 -> lvl0 -- the *_lvl02 gates (include/cufhe_gpu.cuh:332-358,
 *              src/cufhe_gates_gpu.cu:826-979).  Needs cufhe_initialize_lvl02();
 *              always the FP64 FFNT form. */
#define CUFHE_LVL02 2

/* ---- external-product precision form -------------------------------- */
#define CUFHE_FP64_FFNT 0  /* the reference's FP64 negacyclic FFNT */
#define CUFHE_INT8_EXACT 1 /* exact INT8 tensor-core Toeplitz products */

/* Evaluation key in TFHEpp layouts (stands in for TFHEpp::EvalKey):
 *   bk : keybundle == 0 -> TRGSW<lvl1>[636]     (20,840,448 words)
 *        keybundle == 1 -> TRGSW<lvl1>[318][3]  (31,260,672 words),
 *        elements (s0 s1, s0 (1-s1), (1-s0) s1) of each key pair
 *   ksk: TLWE<lvl0>[1024][7][2]                 (9,132,032 words)  */
typedef struct cufhe_keyview {
    const uint32_t* bk;
    size_t bk_words;
    const uint32_t* ksk;
    size_t ksk_words;
    int keybundle;
} cufhe_keyview;

/* lvl02 evaluation key (stands in for the EvalKey members that
 * Initialize_lvl02 reads, src/cufhe_gates_gpu.cu:75-90):
 *   bk : keybundle == 0 -> TRGSW<lvl2>[636]     (20,840,448 uint64 words)
 *        keybundle == 1 -> TRGSW<lvl2>[318][3]  (31,260,672 uint64 words)
 *   ksk: TLWE<lvl0>[2048][7][2] (lvl20 key switching, 18,264,064 words) */
typedef struct cufhe_keyview02 {
    const uint64_t* bk;
    size_t bk_words;
    const uint32_t* ksk;
    size_t ksk_words;
    int keybundle;
} cufhe_keyview02;

typedef struct cufhe_stream_s* cufhe_stream_t; /* NULL = legacy default stream */

/* ---- setup / teardown ----------------------------------------------- */
/* SetGPUNum(int) -- include/cufhe_gpu.cuh:52, src/cufhe_gates_gpu.cu:38 */
int cufhe_set_gpu_num(int n);
int cufhe_get_gpu_num(void);

/* Initialize(const TFHEpp::EvalKey&) -- src/cufhe_gates_gpu.cu:42-61:
 * uploads the keys to every GPU and converts the bootstrapping key to the
 * forms both precision paths use. */
int cufhe_initialize(const cufhe_keyview* ek);

/* CleanUp() -- src/cufhe_gates_gpu.cu:63-73 */
int cufhe_cleanup(void);

/* Initialize_lvl02(const TFHEpp::EvalKey&, const TFHEpp::SecretKey&) --
 * include/cufhe_gpu.cuh:59, src/cufhe_gates_gpu.cu:75-90: uploads the lvl02
 * keys to every GPU (independent of cufhe_initialize).  CleanUp_lvl02() --
 * include/cufhe_gpu.cuh:64. */
int cufhe_initialize_lvl02(const cufhe_keyview02* ek);
int cufhe_cleanup_lvl02(void);

/* Synchronize() -- include/cufhe_gpu.cuh:70-76 */
int cufhe_synchronize(void);

/* Chooses the external-product form used by subsequent gate calls (the
 * reference fixes it at compile time: CMakeLists.txt:49-62), at lvl1 and at
 * lvl02 alike.  INT8_EXACT needs a bootstrapping key without KeyBundle at
 * the level it runs (lvl1 keys for lvl0/lvl1 gates, lvl02 keys for lvl02
 * gates, circuit bootstrapping and cufhe_blind_rotate_lvl02). */
int cufhe_set_precision(int form);
int cufhe_get_precision(void);

/* ---- streams (class Stream, include/cufhe_gpu.cuh:162-199) ----------- */
/* device < 0 picks GPUs round robin, like Stream() */
int cufhe_stream_create(cufhe_stream_t* st, int device);
int cufhe_stream_destroy(cufhe_stream_t st);
/* StreamQuery(Stream) -- src/cufhe_gates_gpu.cu:104-114: 1 idle, 0 busy */
int cufhe_stream_query(cufhe_stream_t st);
int cufhe_stream_device(cufhe_stream_t st);
int cufhe_stream_synchronize(cufhe_stream_t st);
/* The CUDA stream (cudaStream_t) behind st, for interoperation (events,
 * other libraries' work ordered with the engine's); NULL = legacy default. */
int cufhe_stream_cuda(cufhe_stream_t st, void** cuda_stream);

/* ---- ciphertext buffers (Ctxt's per-GPU device buffer and pinned host
 *      copy: include/cufhe_gpu.cuh:78-121, 203-217) -------------------- */
int cufhe_ctxt_alloc(void** dptr, size_t bytes, int device);
int cufhe_ctxt_free(void* dptr, int device);
int cufhe_host_register(void* host, size_t bytes);
int cufhe_host_unregister(void* host);
int cufhe_memcpy_h2d(void* dst_dev, const void* src_host, size_t bytes, cufhe_stream_t st);
int cufhe_memcpy_d2h(void* dst_host, const void* src_dev, size_t bytes, cufhe_stream_t st);

/* ---- gates ------------------------------------------------------------ */
/* One gate on device-resident ciphertexts: the reference's g* variants
 * (gNand ... gNMux, gNot, gCopy; src/cufhe_gates_gpu.cu:212-221 and
 * include/cufhe_gpu.cuh:243-249).  in1 is unused by Not/Copy, in2 is used by
 * Mux/NMux only. */
int cufhe_gate(int gate, int level, uint32_t* out, const uint32_t* in0, const uint32_t* in1,
               const uint32_t* in2, cufhe_stream_t st);

/* One gate with host ciphertexts: the copying variants (Nand ... NMux, Not,
 * Copy; src/cufhe_gates_gpu.cu:198-210): inputs are copied host -> device,
 * the gate runs, the output is copied back, all asynchronously on st.
 * *_dev are the device buffers of the same ciphertexts. */
int cufhe_gate_copy(int gate, int level, uint32_t* out_host, uint32_t* out_dev,
                    const uint32_t* in0_host, uint32_t* in0_dev, const uint32_t* in1_host,
                    uint32_t* in1_dev, const uint32_t* in2_host, uint32_t* in2_dev,
                    cufhe_stream_t st);

/* Batched gates (no counterpart in the reference, which launches one kernel
 * per gate): count gates, gate ids in host memory (NULL: every gate is
 * uniform_gate); in0/in1/in2/out are device arrays of count ciphertexts of
 * the given level. */
int cufhe_gate_batch(const int32_t* gates_host, int uniform_gate, size_t count, int level,
                     uint32_t* out, const uint32_t* in0, const uint32_t* in1,
                     const uint32_t* in2, cufhe_stream_t st);

/* Same with host arrays: copies the inputs in, runs, copies the outputs
 * back (asynchronous on st; host arrays should be pinned for overlap). */
int cufhe_gate_batch_host(const int32_t* gates_host, int uniform_gate, size_t count, int level,
                          uint32_t* out_host, const uint32_t* in0_host, const uint32_t* in1_host,
                          const uint32_t* in2_host, cufhe_stream_t st);

/* Batched uniform gates that allocate no device memory.  This entry point
 * has no counterpart in the reference.  It is for callers that cannot let
 * the library allocate: services with a device-memory budget fixed at start,
 * hosts whose own allocator owns all device memory, and latency-critical
 * code that cannot absorb the synchronisation an allocation may cause.
 * cufhe_gate_batch grows a per-stream workspace with cudaMalloc; this one
 * keeps its lane buffers in a fixed array compiled into the library (about
 * 1.7 MB on every GPU that loads it, held until exit) and therefore accepts
 * at most 256 blind rotations per call (256 binary gates or 128 Mux/NMux);
 * larger calls return CUFHE_ERR_ARG.  Only CUFHE_LVL0 and CUFHE_LVL1 are
 * accepted (CUFHE_LVL02 returns CUFHE_ERR_ARG), and it always runs the FP64
 * FFNT form, whatever cufhe_set_precision selected.  Otherwise the arguments
 * are those of cufhe_gate_batch with every gate equal to `gate`; the caller
 * passes device inputs and outputs.  The first call on a device looks up the
 * array's device address, so make it before any stream capture.  All calls
 * share the array: calls whose work overlaps on the GPU race and corrupt
 * each other's results, so keep them on one stream or synchronise between
 * them. */
int cufhe_gate_batch_noalloc(int gate, size_t count, int level, uint32_t* out,
                             const uint32_t* in0, const uint32_t* in1, const uint32_t* in2,
                             cufhe_stream_t st);

/* ---- lower-level path pieces (used by the parity tests) --------------- */
/* Blind rotation of count lvl0 TLWEs (device [count][637]) with test
 * polynomial mu, first `steps` CMUX steps (KeyBundle pairs) when steps >= 0;
 * writes the TRLWE accumulators [count][2][1024] (acc_out, may be NULL) and
 * the SampleExtract results [count][1025] (tlwe_out, may be NULL).
 * __BlindRotate__ / __SampleExtractIndex__, include/gatebootstrapping_gpu.cuh
 * :801-884, :1335-1380, src/bootstrap_gpu.cu:1201-1221. */
int cufhe_blind_rotate(const uint32_t* tlwe0, size_t count, uint32_t mu, int steps,
                       uint32_t* acc_out, uint32_t* tlwe_out, cufhe_stream_t st);

/* Identity key switching lvl1 -> lvl0 of count TLWEs (device arrays):
 * KeySwitchFromTLWE, include/keyswitch_gpu.cuh:128-187; SEIandKS,
 * src/keyswitch_gpu.cu:52-68. */
int cufhe_identity_keyswitch(const uint32_t* tlwe1, size_t count, uint32_t* tlwe0_out,
                             cufhe_stream_t st);

/* lvl02 counterparts: blind rotation of count lvl0 TLWEs to lvl2 with test
 * polynomial mu (Torus64, 2^61 for the gates), first `steps` steps when
 * steps >= 0; acc_out: TRLWE<lvl2> [count][2][2048], tlwe2_out: TLWE<lvl2>
 * [count][2049] (uint64 words, device memory, either may be NULL). */
int cufhe_blind_rotate_lvl02(const uint32_t* tlwe0, size_t count, uint64_t mu, int steps,
                             uint64_t* acc_out, uint64_t* tlwe2_out, cufhe_stream_t st);

/* Key switching lvl2 -> lvl0 of count TLWE<lvl2> (uint64 [count][2049]) into
 * TLWE<lvl0> (KeySwitchFromTLWE<lvl20param>, include/keyswitch_gpu.cuh:128-187). */
int cufhe_identity_keyswitch_lvl20(const uint64_t* tlwe2, size_t count, uint32_t* tlwe0_out,
                                   cufhe_stream_t st);

/* ---- circuits of dependent gates -------------------------------------- */
/* No counterpart in the reference, whose callers track dependencies
 * themselves (polling StreamQuery per gate, test/test_intensive.cc:23-56).
 *
 * A circuit is a DAG of gates over a table of num_wires ciphertexts of one
 * level (CUFHE_LVL0, CUFHE_LVL1 or CUFHE_LVL02): gate g computes
 * gate_ops[g] on wires in0[g] (, in1[g], in2[g] as the gate needs; Mux takes
 * in0 = selector, in1 = selected when 1, in2 = selected when 0) and writes wire
 * out[g].  Every wire is written by at most one gate; wires no gate writes are
 * the circuit's inputs.  Gates may be listed in any order.
 *
 * cufhe_circuit_create checks the DAG (ranges, single assignment, no cycle),
 * levelises it into waves of independent gates (a gate's wave is one more than
 * the latest wave among the gates it reads from), moves gates with slack out
 * of waves wider than one resident round of blind rotations (4 x SMs lanes at
 * lvl0/lvl1, 2 x SMs at lvl02) into later narrow waves without adding waves,
 * uploads every wave's plan and wire indices once and sizes a private
 * workspace for the widest wave.  cufhe_circuit_plan runs the same checks,
 * levelisation and balancing on the host only (no GPU, no keys) for a given
 * SM count (<= 0: 148) and returns each gate's wave.
 * cufhe_circuit_run runs all waves in order on `st` over the device wire
 * table `wires` ([num_wires][words of the level]); with use_graph = 1 the
 * waves are captured into one CUDA graph the first time (and again when
 * `wires` or the precision form changes) and replayed afterwards, in either
 * precision form.  Runs of one circuit share its workspace: do not overlap
 * them on the GPU.  Per-kernel profiling does not see graph replays. */
typedef struct cufhe_circuit_s* cufhe_circuit_t;
int cufhe_circuit_create(cufhe_circuit_t* c, int level, size_t num_wires, size_t num_gates,
                         const int32_t* gate_ops, const int32_t* in0, const int32_t* in1,
                         const int32_t* in2, const int32_t* out, int device);
int cufhe_circuit_plan(int level, size_t num_wires, size_t num_gates, const int32_t* gate_ops,
                       const int32_t* in0, const int32_t* in1, const int32_t* in2,
                       const int32_t* out, int sms, int32_t* wave_of_gate, int* num_waves);
int cufhe_circuit_info(cufhe_circuit_t c, int* waves, int* max_wave_gates, int* max_wave_lanes);
/* gates and blind rotations of each wave; returns the number of waves */
int cufhe_circuit_wave_sizes(cufhe_circuit_t c, int32_t* gates, int32_t* lanes, size_t cap);
int cufhe_circuit_run(cufhe_circuit_t c, uint32_t* wires, cufhe_stream_t st, int use_graph);
int cufhe_circuit_destroy(cufhe_circuit_t c);

/* A circuit whose connected components (gates joined through the wires one
 * writes and another reads) are packed into up to `parts` groups with
 * balanced blind rotations, each group planned into waves and run on a
 * stream of its own: cufhe_circuit_run forks from `st` into the groups'
 * streams and joins back, so that one group's partly filled last round of
 * rotations in a wave overlaps the other groups' waves.  Results are
 * bit-identical to cufhe_circuit_create's.  With one component (or
 * parts = 1) it is cufhe_circuit_create.  cufhe_circuit_info reports the
 * most waves of any group; cufhe_circuit_wave_sizes the gates and rotations
 * of the groups' wave w together.  cufhe_circuit_split_plan returns the
 * group of every gate (host only, no GPU) and the number of groups.
 * Every group keeps a workspace of its own, sized for its widest wave (the
 * INT8 form's part on the group's first INT8 run, zeroed on the group's
 * stream), so device memory grows with the number of groups.
 * parts: 1 .. 64. */
int cufhe_circuit_create_split(cufhe_circuit_t* c, int level, size_t num_wires,
                               size_t num_gates, const int32_t* gate_ops, const int32_t* in0,
                               const int32_t* in1, const int32_t* in2, const int32_t* out,
                               int device, int parts);
int cufhe_circuit_split_plan(int level, size_t num_wires, size_t num_gates,
                             const int32_t* gate_ops, const int32_t* in0, const int32_t* in1,
                             const int32_t* in2, const int32_t* out, int parts,
                             int32_t* group_of_gate);

/* ---- one batch or one circuit over several GPUs -------------------------
 * The reference spreads work over GPUs only through the device each Stream
 * is given in turn, with the keys replicated on every GPU
 * (include/cufhe_gpu.cuh:164-175, src/cufhe_gates_gpu.cu:38-61); that stays
 * available here (cufhe_stream_create with device -1).  These entry points
 * split ONE batch or ONE circuit over `shards` shards (<= 0: the
 * cufhe_set_gpu_num count, at most 64); shard s runs on device
 * s % cufhe_set_gpu_num, each with its own key replica.  Gates are
 * independent, so a batch needs no data exchange: it splits into contiguous
 * gate ranges with balanced blind-rotation lanes.  A circuit splits every
 * wave (lanes balanced per wave; a gate preferably joins the shard that wrote
 * its operands), and each wire that one shard writes and another reads later
 * is copied into the reader's own wire table right after the wave that
 * writes it (the writer's device stores into the peer's memory; peer access
 * is enabled between the devices in use).
 *
 * cufhe_batch_shard_plan: host only; bounds[0..shards] with shard k holding
 * gates [bounds[k], bounds[k + 1]).
 * cufhe_gate_batch_sharded_host: cufhe_gate_batch_host split that way, each
 * shard on an engine stream of its device; returns when all shards are done.
 * cufhe_circuit_shard_plan: host only (no GPU, no keys); the waves of
 * cufhe_circuit_plan, a shard per gate, and the number of wire copies.
 * cufhe_sharded_create: the same plan on the devices (keys initialised on
 * each device in use).  cufhe_sharded_run(c, wires): wires[s] is shard s's
 * wire table [num_wires][words] on its device (cufhe_sharded_device); the
 * circuit's input wires must be in every shard's table before the call.  The
 * run is asynchronous; after it each shard's table holds the wires its gates
 * wrote and the wires it received.  cufhe_sharded_collect(c, wires, dst)
 * copies every gate output into shard dst's table; cufhe_sharded_synchronize
 * waits for both.  Runs of one sharded circuit must not overlap. */
typedef struct cufhe_sharded_s* cufhe_sharded_t;
int cufhe_batch_shard_plan(const int32_t* gates_host, int uniform_gate, size_t count, int shards,
                           size_t* bounds);
int cufhe_gate_batch_sharded_host(const int32_t* gates_host, int uniform_gate, size_t count,
                                  int level, uint32_t* out_host, const uint32_t* in0_host,
                                  const uint32_t* in1_host, const uint32_t* in2_host, int shards);
int cufhe_circuit_shard_plan(int level, size_t num_wires, size_t num_gates, const int32_t* gate_ops,
                             const int32_t* in0, const int32_t* in1, const int32_t* in2,
                             const int32_t* out, int sms, int shards, int32_t* wave_of_gate,
                             int32_t* shard_of_gate, int* num_waves, size_t* num_copies);
int cufhe_sharded_create(cufhe_sharded_t* c, int level, size_t num_wires, size_t num_gates,
                         const int32_t* gate_ops, const int32_t* in0, const int32_t* in1,
                         const int32_t* in2, const int32_t* out, int shards);
int cufhe_sharded_info(cufhe_sharded_t c, int* waves, size_t* copies, int* shards);
/* device of a shard (or a negative error code) */
int cufhe_sharded_device(cufhe_sharded_t c, int shard);
int cufhe_sharded_run(cufhe_sharded_t c, uint32_t* const* wires);
int cufhe_sharded_collect(cufhe_sharded_t c, uint32_t* const* wires, int dst);
int cufhe_sharded_synchronize(cufhe_sharded_t c);
int cufhe_sharded_destroy(cufhe_sharded_t c);

/* ---- circuit bootstrapping, CMUX, lookup tables ----------------------- */
/* Gadgets of TRGSW<lvl1> (N = 1024, Torus32): */
#define CUFHE_GADGET_LVL1 0 /* l = 2, Bgbit = 8: the bootstrapping gadget (lvl1param) */
#define CUFHE_GADGET_CB 1   /* l = 3, Bgbit = 6: circuit-bootstrapping output */

/* Keys of circuit bootstrapping (CGGI17 form): the two private key-switching
 * keys lvl2 -> lvl1 (basebit 4, t 10), each TRLWE<lvl1>[2049][10][15] =
 * 629,452,800 uint32 words, encrypting f(k_i (u+1) 2^-4(j+1)) with
 * f(x) = -x s1 (privks0, rows carrying the message in the mask) and f(x) = x
 * (privks1).  Circuit bootstrapping also needs cufhe_initialize_lvl02 (its
 * blind rotations go to lvl2).  No counterpart in the reference, whose circuit
 * bootstrapping is annihilation-based (include/circuitbootstrapping_gpu.cuh:
 * 1-69) and takes different keys. */
typedef struct cufhe_cbkeyview {
    const uint32_t* privks0;
    const uint32_t* privks1;
    size_t words; /* of each key */
} cufhe_cbkeyview;
int cufhe_initialize_cb(const cufhe_cbkeyview* kv);
int cufhe_cleanup_cb(void);

/* Private key switching of count TLWE<lvl2> (uint64 [count][2049], device)
 * with key func (0 or 1) into TRLWE<lvl1> [count][2][1024] (device). */
int cufhe_private_keyswitch(const uint64_t* tlwe2, size_t count, int func, uint32_t* trlwe_out,
                            cufhe_stream_t st);

/* Circuit bootstrapping of count lvl0 TLWEs (device [count][637], bits
 * encrypted as +-1/8) into TRGSW<lvl1> with the CB gadget, raw Torus32
 * [count][6 rows][2][1024] (row r = j*3 + i): per bit three blind rotations
 * to lvl2 with test polynomial 2^-(6(i+1)+1), plus that value on b, then
 * private key switching with privks0 (rows j = 0) and privks1 (rows j = 1). */
int cufhe_circuit_bootstrap(const uint32_t* tlwe0, size_t count, uint32_t* trgsw_out,
                            cufhe_stream_t st);

/* Raw TRGSW<lvl1> ([count][2l][2][1024]) -> Fourier form ([count][2l][2][512]
 * complex doubles, interleaved re/im) for cufhe_cmux / cufhe_lut_eval
 * (the reference's TRGSW NTT form, src/bootstrap_gpu.cu:59-112). */
int cufhe_trgsw_to_fft(int gadget, const uint32_t* trgsw, size_t count, double* fft_out,
                       cufhe_stream_t st);

/* Batched CMUX: out[i] = d0[i] + ExtProd(C_i, d1[i] - d0[i]) over TRLWE<lvl1>
 * (device [count][2][1024]) with Fourier TRGSWs C_i -- CMUXNTT
 * (src/cufhe_gates_gpu.cu:116-133) for count selections at once. */
int cufhe_cmux(int gadget, const double* trgsw_fft, const uint32_t* d1, const uint32_t* d0,
               uint32_t* out, size_t count, cufhe_stream_t st);

/* 8-bit -> 8-bit lookup tables: luts_host [num_luts][256] bytes (entry x
 * holds the 8 output bits of input x); trgsw_fft [num_luts][8] Fourier
 * TRGSWs with the CB gadget (TRGSW k of a table selects on input bit k,
 * least significant first: e.g. circuit-bootstrapped bits); out
 * [num_luts][8][1025] TLWE<lvl1> (device) encrypting output bit b as +-mu.
 * Each table is a CMUX tree of 255 CMUXes over leaves packing the 8 output
 * bits in coefficients 0..7; the trees of all tables advance level by level. */
int cufhe_lut_eval(const uint8_t* luts_host, size_t num_luts, const double* trgsw_fft,
                   uint32_t mu, uint32_t* tlwe1_out, cufhe_stream_t st);

/* ---- autotuner -------------------------------------------------------- */
/* Measures, on the current device with its keys, how many lanes (blind
 * rotations) per CTA the FP64 blind rotation should carry for a ladder of
 * batch sizes, and makes every later launch on that device use the
 * measured choice (takes about a second; CUFHE_BR_LANES_PER_CTA still
 * overrides).  cufhe_autotune_table reads the table back: batches of up to
 * lanes[i] blind rotations use lanes_per_cta[i]; returns its length (0 when
 * the device is untuned and a built-in rule applies). */
int cufhe_autotune(void);
int cufhe_autotune_table(int32_t* lanes, int32_t* lanes_per_cta, int cap);

/* ---- diagnostics ----------------------------------------------------- */
/* Per-kernel timing: when enabled, every engine kernel launch is bracketed
 * by CUDA events on its stream; cufhe_profile_read() sums the durations of
 * one kernel class (waits for the recorded events).  Classes: */
#define CUFHE_K_IKS 0        /* identity key switching */
#define CUFHE_K_PREADD 1     /* lvl0 pre-add (BR->IKS order) */
#define CUFHE_K_BR_FP64 2    /* FP64 FFNT blind rotation + SampleExtract */
#define CUFHE_K_BR_INT8 3    /* INT8 exact blind rotation step kernels */
#define CUFHE_K_FINALIZE 4   /* lane combination (Mux) and Not/Copy */
#define CUFHE_K_BR_FP64_LVL02 5 /* FP64 FFNT blind rotation to lvl2 + SampleExtract */
#define CUFHE_K_IKS_LVL20 6  /* key switching lvl2 -> lvl0 */
#define CUFHE_K_PRIVKS 7     /* private key switching lvl2 -> lvl1 */
#define CUFHE_K_CMUX 8       /* CMUX (lookup tables, cufhe_cmux) */
#define CUFHE_K_BR_INT8_LVL02 9 /* INT8 exact blind rotation to lvl2 step kernels */
#define CUFHE_K_CLASSES 10
int cufhe_profile_enable(int on);
int cufhe_profile_reset(void);
int cufhe_profile_read(int kernel_class, double* total_ms, uint64_t* launches);
/* FP64 FMA throughput of the current device in TFLOP/s (roof of the FFNT
 * path; runs a short probe kernel) */
int cufhe_measure_fp64_peak(double* tflops);
/* Failure-path self-test (no GPU fault): launches a kernel whose bounded
 * mbarrier wait runs out (a barrier nothing arrives at, about 1 ms of polls),
 * so it sets the device error flag exactly as a tensor-core kernel whose wait
 * gave up; then reports like cufhe_synchronize.  Returns CUFHE_ERR_CUDA (the
 * timeout was detected and the flag cleared) on a healthy engine; the CUDA
 * context stays usable.  Needs cufhe_initialize. */
int cufhe_selftest_wait_timeout(void);
/* INT8 tensor-core throughput of the current device in TOP/s: back-to-back
 * tcgen05.mma.kind::i8 M128 N256 K32 with random operands on every SM (roof
 * of the exact path's step GEMM; runs a short probe kernel) */
int cufhe_measure_int8_peak(double* tops);

const char* cufhe_last_error(void);
/* kernels launched by this process so far (all devices) */
uint64_t cufhe_kernel_launches(void);
/* 1 when the library was built for sm_100a and a device is visible */
int cufhe_device_ok(void);

#ifdef __cplusplus
}
#endif

#endif /* CUFHE_B200_H */
