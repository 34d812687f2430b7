// Instantiates the streaming forward kernels (gb_stream.cuh).
#include "gb_kernels.h"
#include "gb_stream.cuh"

#include <cuda_runtime.h>

namespace gb {
namespace host {
namespace {

template <int R>
void *pick(bool en, int img)
{
    if (img == 1) return en ? (void *)&fwd_stream_kernel<R, true, 1> : (void *)&fwd_stream_kernel<R, false, 1>;
    if (img == 2) return en ? (void *)&fwd_stream_kernel<R, true, 2> : (void *)&fwd_stream_kernel<R, false, 2>;
    return en ? (void *)&fwd_stream_kernel<R, true, 0> : (void *)&fwd_stream_kernel<R, false, 0>;
}

}  // namespace

StepKernel fwd_stream_kernel_for(int R, bool en, int img)
{
    StepKernel k;
    k.fn = R == 2 ? pick<2>(en, img) : R == 4 ? pick<4>(en, img) : nullptr;
    k.smem = kStreamSmemBytes;
    k.stream = true;
    return k;
}

}  // namespace host
}  // namespace gb
