// Instantiates the resident forward kernels (gb_resident.cuh) for each tile
// height: 4 warps for 4-row tiles, 8 for 8 and 12, 12 for 36, 16 otherwise
// (measured against one boundary item per thread and two interior rows per
// warp, which ran 7 % slower on the 400 x 1200 grid and 26 % on 100 x 200
// with 8-row tiles); each with the exchange through global memory ((value,
// tag) words), and through distributed shared memory within a cluster; and
// the one-exchange-a-step kernels (gb_resident_sx.cuh, 4th order).
#include "gb_kernels.h"
#include "gb_resident.cuh"
#include "gb_resident_sx.cuh"

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
    k.tile_words = (size_t)kResParts * G::PART;
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

template <int NW, int TZ>
ResidentKernel make_sx()
{
    using G = SxGeo<NW, TZ>;
    ResidentKernel k;
    k.fn = (void *)&resident_sx_kernel<NW, TZ>;
    k.smem = G::SMEM;
    k.threads = G::NTH;
    k.tile_words = 2 * (size_t)G::SLOT;
    return k;
}

// one exchange a step: 8 warps up to 16-row tiles, 16 above
ResidentKernel pick_sx(int tz)
{
    switch (tz) {
    case 4: return make_sx<8, 4>();
    case 8: return make_sx<8, 8>();
    case 12: return make_sx<8, 12>();
    case 16: return make_sx<8, 16>();
    case 24: return make_sx<16, 24>();
    case 32: return make_sx<16, 32>();
    case 36: return make_sx<16, 36>();
    case 40: return make_sx<16, 40>();
    default: return ResidentKernel{};
    }
}

}  // namespace

ResidentKernel resident_kernel(int R, int tz, int exchange)
{
    if (exchange == 2) return R == 2 ? pick_sx(tz) : ResidentKernel{};
    const bool cluster = exchange == 1;
    if (R == 2) return cluster ? pick<2, true>(tz) : pick<2, false>(tz);
    if (R == 4) return cluster ? pick<4, true>(tz) : pick<4, false>(tz);
    return ResidentKernel{};
}

}  // namespace host
}  // namespace gb
