// Instantiates the batched forward step kernels (gb_batch.cuh), 16-row tiles
// (the adjoint ones: gb_pick_batch_adj.cu).
#include "gb_batch.cuh"
#include "gb_kernels.h"

#include <cuda_runtime.h>

namespace gb {
namespace host {
namespace {

template <int R, bool FS>
void *pick_fwd(bool en, int img)
{
    if (img == 1) return en ? (void *)&fwd_batch_kernel<R, 16, FS, true, 1> : (void *)&fwd_batch_kernel<R, 16, FS, false, 1>;
    if (img == 2) return en ? (void *)&fwd_batch_kernel<R, 16, FS, true, 2> : (void *)&fwd_batch_kernel<R, 16, FS, false, 2>;
    return en ? (void *)&fwd_batch_kernel<R, 16, FS, true, 0> : (void *)&fwd_batch_kernel<R, 16, FS, false, 0>;
}

}  // namespace

StepKernel fwd_batch_kernel_for(int R, bool fs, bool en, int img)
{
    StepKernel k;
    if (R == 2) {
        k.fn = fs ? pick_fwd<2, true>(en, img) : pick_fwd<2, false>(en, img);
        k.smem = fwd_smem_bytes<2, 16>();
    } else if (R == 4) {
        k.fn = fs ? pick_fwd<4, true>(en, img) : pick_fwd<4, false>(en, img);
        k.smem = fwd_smem_bytes<4, 16>();
    }
    return k;
}

}  // namespace host
}  // namespace gb
