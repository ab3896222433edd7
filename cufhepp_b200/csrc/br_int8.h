// Exact INT8 tensor-core blind rotation (tcgen05, sm_100a): key and
// workspace types shared with the engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cufhe {

struct Int8Key {
    bool ready = false;
    bool kb = false;           // KeyBundle key: TRGSW[n0 / 2][3], one step per pair
    uint8_t* limbs = nullptr;  // per TRGSW: Toeplitz source rows of the key limbs
    size_t bytes = 0;
};

struct Int8Workspace {
    size_t cap = 0;       // lanes
    uint32_t* acc = nullptr;
    int8_t* digits = nullptr;
    uint16_t* abar = nullptr;
};

// lvl0 -> lvl2 form (N = 2048, l = 4, Bgbit = 10, Torus64): eight key limbs,
// two digit limbs
struct Int8Workspace2 {
    size_t cap = 0;       // lanes
    uint64_t* acc = nullptr;
    int8_t* digits = nullptr;
    uint16_t* abar = nullptr;
};

// bk_dev: BootstrappingKey<lvl01> in the TFHEpp layout, plain TRGSW[636] or
// (kb) KeyBundle TRGSW[318][3]
cudaError_t int8_key_build(Int8Key& k, const uint32_t* bk_dev, bool kb, cudaStream_t st);
void int8_key_free(Int8Key& k);
void int8_workspace_free(Int8Workspace& w);
// The launchers are asynchronous (stream-ordered, capturable into a CUDA
// graph once the workspace is reserved): a kernel whose bounded wait gives
// up sets *err, which the caller reads at synchronisation.
// int8_reserve*: size the workspace for `lanes` and set the kernels'
// attributes; call before a graph capture.  A new workspace is zeroed on
// `st`, so the launches that use it must be ordered after that stream's work.
// launch_br_int8: `steps` counts CMUX steps of a plain key, pairs of a
// KeyBundle key (all of them when steps < 0).
cudaError_t int8_reserve(Int8Workspace& w, int lanes, cudaStream_t st);
cudaError_t int8_reserve2(Int8Workspace2& w, int lanes, cudaStream_t st);
cudaError_t launch_br_int8(const Int8Key& k, Int8Workspace& w, const uint32_t* lane_in, int lanes,
                           uint32_t mu, int steps, uint32_t* acc_out, uint32_t* lane_out,
                           int* err, cudaStream_t st, int* launches);

// bk2_dev: BootstrappingKey<lvl02>, plain TRGSW<lvl2>[636] or (kb) KeyBundle
// TRGSW<lvl2>[318][3]; launch_br2_int8's `steps` counts CMUX steps or pairs
cudaError_t int8_key2_build(Int8Key& k, const uint64_t* bk2_dev, bool kb, cudaStream_t st);
void int8_workspace2_free(Int8Workspace2& w);
cudaError_t launch_br2_int8(const Int8Key& k, Int8Workspace2& w, const uint32_t* lane_in, int lanes,
                            uint64_t mu, int steps, uint64_t* acc_out, uint64_t* lane_out,
                            int* err, cudaStream_t st, int* launches);

}  // namespace cufhe
