// Instantiates the resident forward kernels (gb_resident.cuh) for each tile
// height: 4 warps for 4-row tiles, 8 for 8 and 12, 12 for 36, 16 otherwise.
#include "gb_kernels.h"
#include "gb_resident.cuh"

#include <cuda_runtime.h>

namespace gb {
namespace host {
namespace {

template <int R, int NW, int TZ>
ResidentKernel make()
{
    using G = ResGeo<R, NW, TZ>;
    ResidentKernel k;
    k.fn = (void *)&resident_fwd_kernel<R, NW, TZ>;
    k.smem = G::SMEM;
    k.threads = G::NTH;
    k.part_floats = G::PART;
    return k;
}

template <int R>
ResidentKernel pick(int tz)
{
    switch (tz) {
    case 4: return make<R, 4, 4>();
    case 8: return make<R, 8, 8>();
    case 12: return make<R, 8, 12>();
    case 16: return make<R, 16, 16>();
    case 24: return make<R, 16, 24>();
    case 32: return make<R, 16, 32>();
    case 36: return make<R, 12, 36>();
    case 40: return make<R, 16, 40>();
    case 48: return make<R, 16, 48>();
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
