// Instantiates the resident forward kernels (gb_resident.cuh) for each tile
// height: 4 warps for 4-row tiles, 8 for 8 and 12, 12 for 36, 16 otherwise
// (measured against one boundary item per thread and two interior rows per
// warp, which ran 7 % slower on the 400 x 1200 grid and 26 % on 100 x 200
// with 8-row tiles); each with the exchange through global memory ((value,
// tag) words), and through distributed shared memory within a cluster.
#include "gb_kernels.h"
#include "gb_resident.cuh"

#include <cuda_runtime.h>

namespace gb {
namespace host {
namespace {

template <int R, int NW, int TZ, bool CL>
ResidentKernel make()
{
    using G = ResGeo<R, NW, TZ>;
    ResidentKernel k;
    k.fn = (void *)&resident_fwd_kernel<R, NW, TZ, CL>;
    k.smem = G::SMEM;
    k.threads = G::NTH;
    k.part_words = G::PART;
    return k;
}

template <int R, bool CL>
ResidentKernel pick(int tz)
{
    switch (tz) {
    case 4: return make<R, 4, 4, CL>();
    case 8: return make<R, 8, 8, CL>();
    case 12: return make<R, 8, 12, CL>();
    case 16: return make<R, 16, 16, CL>();
    case 24: return make<R, 16, 24, CL>();
    case 32: return make<R, 16, 32, CL>();
    case 36: return make<R, 12, 36, CL>();
    case 40: return make<R, 16, 40, CL>();
    default: return ResidentKernel{};
    }
}

}  // namespace

ResidentKernel resident_kernel(int R, int tz, bool cluster)
{
    if (R == 2) return cluster ? pick<2, true>(tz) : pick<2, false>(tz);
    if (R == 4) return cluster ? pick<4, true>(tz) : pick<4, false>(tz);
    return ResidentKernel{};
}

}  // namespace host
}  // namespace gb
