// Instantiates the adjoint tile step kernels of stencil half-width 4.
#include "gb_adj.cuh"
#include "gb_kernels.h"

#include <cuda_runtime.h>

namespace gb {
namespace host {
namespace {

template <int TZ, int IMGF>
void *pick_f(bool fs, bool rho)
{
    if (fs) return rho ? (void *)&adj_step_kernel<4, TZ, true, true, IMGF> : (void *)&adj_step_kernel<4, TZ, true, false, IMGF>;
    return rho ? (void *)&adj_step_kernel<4, TZ, false, true, IMGF> : (void *)&adj_step_kernel<4, TZ, false, false, IMGF>;
}

}  // namespace

// The default 16-row tiles get one kernel per imaging format (the loads are
// issued early, ahead of the stage wait, and a format switch there costs);
// the 32-row tiles read the format at run time.
StepKernel adj_tile_kernel_r4(int tz, bool fs, bool rho, int img_fmt)
{
    StepKernel k;
    if (tz == 16) {
        k.fn = img_fmt == kImgBF16 ? pick_f<16, kImgBF16>(fs, rho)
             : img_fmt == kImgF24  ? pick_f<16, kImgF24>(fs, rho)
                                   : pick_f<16, kImgF32>(fs, rho);
        k.smem = adj_smem_bytes<4, 16>();
    } else if (tz == 32) {
        k.fn = pick_f<32, -1>(fs, rho);
        k.smem = adj_smem_bytes<4, 32>();
    }
    return k;
}

}  // namespace host
}  // namespace gb
