// Stencil evaluation on the shared-memory rectangles, shared by the forward
// and adjoint step kernels.  Each lane owns 4 adjacent columns; the
// z-direction taps come from a per-warp register window.  Every tap is an
// explicit fused multiply-add, so every kernel that inlines these rounds the
// same way.
#pragma once

#include "gb_device.cuh"

namespace gb {

// Divergence of a staggered velocity pair at 4 adjacent cells of one row of
// the p rectangle (reference order acoustic_2d.py:216-225):
//   D[q] = sum_k c_k * (((vx[j+k] - vx[j-1-k]) + vz[i+k]) - vz[i-1-k])
// vxr: the row of the vx rectangle (136 wide, column 0 = x0 - 8); the lane's
// first column j = x0 - 4 + 4*lane sits at vxr[4*lane + 4].  wz: window of
// vz rows with wz[u + R] = row i.
template <int R>
__device__ __forceinline__ void divergence4(const float *vxr, int lane, const float4 *wz, int u,
                                            const float (&c)[4], float (&D)[4])
{
    float e[12];
    {
        const float4 e0 = lds4(vxr + 4 * lane);
        const float4 e1 = lds4(vxr + 4 * lane + 4);
        const float4 e2 = lds4(vxr + 4 * lane + 8);
        e[0] = e0.x; e[1] = e0.y; e[2] = e0.z; e[3] = e0.w;
        e[4] = e1.x; e[5] = e1.y; e[6] = e1.z; e[7] = e1.w;
        e[8] = e2.x; e[9] = e2.y; e[10] = e2.z; e[11] = e2.w;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float d = 0.f;
#pragma unroll
        for (int k = 0; k < R; ++k)
            d = __fmaf_rn(c[k], ((e[q + 4 + k] - e[q + 3 - k]) + at(wz[u + R + k], q)) - at(wz[u + R - 1 - k], q), d);
        D[q] = d;
    }
}

// The two parts of divergence4 kept apart (the CPML option needs each one):
//   Dx[q] = sum_k c_k (vx[j+k] - vx[j-1-k]),  Dz[q] = sum_k c_k (vz[i+k] - vz[i-1-k])
template <int R>
__device__ __forceinline__ void divergence4_split(const float *vxr, int lane, const float4 *wz, int u,
                                                  const float (&c)[4], float (&Dx)[4], float (&Dz)[4])
{
    float e[12];
    {
        const float4 e0 = lds4(vxr + 4 * lane);
        const float4 e1 = lds4(vxr + 4 * lane + 4);
        const float4 e2 = lds4(vxr + 4 * lane + 8);
        e[0] = e0.x; e[1] = e0.y; e[2] = e0.z; e[3] = e0.w;
        e[4] = e1.x; e[5] = e1.y; e[6] = e1.z; e[7] = e1.w;
        e[8] = e2.x; e[9] = e2.y; e[10] = e2.z; e[11] = e2.w;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float dx = 0.f, dz = 0.f;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            dx = __fmaf_rn(c[k], e[q + 4 + k] - e[q + 3 - k], dx);
            dz = __fmaf_rn(c[k], at(wz[u + R + k], q) - at(wz[u + R - 1 - k], q), dz);
        }
        Dx[q] = dx;
        Dz[q] = dz;
    }
}

// x-derivative of p at the staggered vx points of 4 adjacent cells:
//   D[q] = sum_k c_k (p[j+1+k] - p[j-k])        (acoustic_2d.py:248-252)
// pr: the row of the p rectangle (128 wide, column 0 = x0 - 4); the lane's
// first column j sits at pr[4*lane].
template <int R>
__device__ __forceinline__ void grad_x4(const float *pr, int lane, const float (&c)[4], float (&D)[4], float4 &mid)
{
    float f[12];
    {
        const float4 f0 = lds4(pr + 4 * lane - 4);
        const float4 f1 = lds4(pr + 4 * lane);
        const float4 f2 = lds4(pr + 4 * lane + 4);
        f[0] = f0.x; f[1] = f0.y; f[2] = f0.z; f[3] = f0.w;
        f[4] = f1.x; f[5] = f1.y; f[6] = f1.z; f[7] = f1.w;
        f[8] = f2.x; f[9] = f2.y; f[10] = f2.z; f[11] = f2.w;
        mid = f1;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float d = 0.f;
#pragma unroll
        for (int k = 0; k < R; ++k) d = __fmaf_rn(c[k], f[q + 5 + k] - f[q + 4 - k], d);
        D[q] = d;
    }
}

// z-derivative of p at the staggered vz points:
//   D[q] = sum_k c_k (p[i+1+k] - p[i-k])        (acoustic_2d.py:260-264)
// wp: window of p rows with wp[u + R] = row i + 1.
template <int R>
__device__ __forceinline__ void grad_z4(const float4 *wp, int u, const float (&c)[4], float (&D)[4])
{
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float d = 0.f;
#pragma unroll
        for (int k = 0; k < R; ++k) d = __fmaf_rn(c[k], at(wp[u + R + k], q) - at(wp[u + R - 1 - k], q), d);
        D[q] = d;
    }
}

// 2-D tiled TMA load of a coefficient plane (Nz x pitch).
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace gb
