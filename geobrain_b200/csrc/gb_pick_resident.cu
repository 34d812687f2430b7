// Instantiates the resident forward kernels (gb_resident.cuh): 8 warps for
// tiles of 8 .. 48 rows (1 .. 6 rows per warp), 16 warps for 32 and 48 rows.
#include "gb_kernels.h"
#include "gb_resident.cuh"

#include <cuda_runtime.h>

namespace gb {
namespace host {
namespace {

template <int R, int NW, int LV>
ResidentKernel make()
{
    using G = ResGeo<R, NW, LV>;
    ResidentKernel k;
    k.fn = (void *)&resident_fwd_kernel<R, NW, LV>;
    k.smem = G::SMEM;
    k.threads = G::NTH;
    k.part_floats = G::PART;
    return k;
}

template <int R>
ResidentKernel pick(int tz)
{
    switch (tz) {
    case 8: return make<R, 8, 1>();
    case 16: return make<R, 8, 2>();
    case 24: return make<R, 8, 3>();
    case 32: return make<R, 16, 2>();
    case 40: return make<R, 8, 5>();
    case 48: return make<R, 16, 3>();
    default: return ResidentKernel{};
    }
}

}  // namespace

ResidentKernel resident_kernel(int R, int tz)
{
    if (R == 2) return pick<2>(tz);
    if (R == 4) return pick<4>(tz);
    return ResidentKernel{};
}

}  // namespace host
}  // namespace gb
