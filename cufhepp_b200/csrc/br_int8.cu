// Exact INT8 tensor-core blind rotation (placeholder until the tcgen05 path).
#include "br_int8.h"

namespace cufhe {

cudaError_t int8_key_build(Int8Key& k, const uint32_t*, cudaStream_t)
{
    k.ready = false;
    return cudaSuccess;
}
void int8_key_free(Int8Key& k) { k = Int8Key(); }
void int8_workspace_free(Int8Workspace& w) { w = Int8Workspace(); }
cudaError_t launch_br_int8(const Int8Key&, Int8Workspace&, const uint32_t*, int, uint32_t, int,
                           uint32_t*, uint32_t*, cudaStream_t, int* launches)
{
    *launches = 0;
    return cudaErrorNotSupported;
}

}  // namespace cufhe
