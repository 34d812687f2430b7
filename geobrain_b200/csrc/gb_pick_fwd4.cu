// Instantiates the forward tile step kernels of stencil half-width 4.
#include "gb_fwd.cuh"
#include "gb_kernels.h"

#include <cuda_runtime.h>

namespace gb {
namespace host {
namespace {

template <int TZ, bool FS>
void *pick(bool en, int img)
{
    if (img == 1) return en ? (void *)&fwd_step_kernel<4, TZ, FS, true, 1> : (void *)&fwd_step_kernel<4, TZ, FS, false, 1>;
    if (img == 2) return en ? (void *)&fwd_step_kernel<4, TZ, FS, true, 2> : (void *)&fwd_step_kernel<4, TZ, FS, false, 2>;
    return en ? (void *)&fwd_step_kernel<4, TZ, FS, true, 0> : (void *)&fwd_step_kernel<4, TZ, FS, false, 0>;
}

}  // namespace

StepKernel fwd_tile_kernel_r4(int tz, bool fs, bool en, int img)
{
    StepKernel k;
    if (tz == 16) {
        k.fn = fs ? pick<16, true>(en, img) : pick<16, false>(en, img);
        k.smem = fwd_smem_bytes<4, 16>();
    } else if (tz == 32) {
        k.fn = fs ? pick<32, true>(en, img) : pick<32, false>(en, img);
        k.smem = fwd_smem_bytes<4, 32>();
    }
    return k;
}

}  // namespace host
}  // namespace gb
