// Host-side helpers shared by the translation units of the C ABI
// (gb_capi.cu, gb_capi3d.cu).
#pragma once

#include "../../include/geobrain_b200.h"

#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstddef>
#include <cstdint>
#include <string>

namespace gb {
namespace host {

// Records msg as this thread's last error (gb_last_error) and returns code.
int fail(int code, const std::string &msg);
// Clears this thread's last error (every C ABI entry point starts with it).
void clear_error();
// cuTensorMapEncodeTiled, looked up once through the runtime's driver entry
// point (GB_E_CUDA if the driver has none).
int tensor_map_encoder(PFN_cuTensorMapEncodeTiled_v12000 *out);

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
inline char *aligned_ws(void *workspace)
{
    return reinterpret_cast<char *>(align256(reinterpret_cast<uintptr_t>(workspace)));
}

}  // namespace host
}  // namespace gb

// Returns GB_E_CUDA (with the call and the CUDA message as the last error)
// from the enclosing function when a CUDA runtime call fails.
#define GB_CUDA(call)                                                                                 \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return gb::host::fail(GB_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
    } while (0)
