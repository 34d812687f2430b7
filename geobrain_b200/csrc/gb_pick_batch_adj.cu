// Instantiates the batched adjoint step kernels (gb_batch.cuh), 16-row
// tiles: one per imaging format, for batches whose models all store the
// same one, and one that reads each model's format at run time.
#include "gb_batch.cuh"
#include "gb_kernels.h"

#include <cuda_runtime.h>

namespace gb {
namespace host {
namespace {

template <int R, bool FS, bool RHO>
void *pick(int imgf)
{
    switch (imgf) {
    case kImgF32: return (void *)&adj_batch_kernel<R, 16, FS, RHO, kImgF32>;
    case kImgBF16: return (void *)&adj_batch_kernel<R, 16, FS, RHO, kImgBF16>;
    case kImgF24: return (void *)&adj_batch_kernel<R, 16, FS, RHO, kImgF24>;
    default: return (void *)&adj_batch_kernel<R, 16, FS, RHO, -1>;
    }
}

template <int R>
void *pick_r(bool fs, bool rho, int imgf)
{
    if (fs) return rho ? pick<R, true, true>(imgf) : pick<R, true, false>(imgf);
    return rho ? pick<R, false, true>(imgf) : pick<R, false, false>(imgf);
}

}  // namespace

StepKernel adj_batch_kernel_for(int R, bool fs, bool rho, int imgf)
{
    StepKernel k;
    if (R == 2) {
        k.fn = pick_r<2>(fs, rho, imgf);
        k.smem = adj_smem_bytes<2, 16>();
    } else if (R == 4) {
        k.fn = pick_r<4>(fs, rho, imgf);
        k.smem = adj_smem_bytes<4, 16>();
    }
    return k;
}

}  // namespace host
}  // namespace gb
