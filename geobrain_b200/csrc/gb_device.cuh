// Device-side building blocks shared by the propagator kernels: tile
// geometry, TMA / mbarrier wrappers (inline PTX, sm_100a), and small vector
// helpers.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace gb {

// ---------------------------------------------------------------------------
// Tile geometry.
//
// A CTA owns an output tile of TZ rows x TX = 120 columns of one model and
// walks a group of shots through it.  For each shot it stages three halo
// rectangles of the current state in shared memory with TMA:
//
//   sP   pressure     rows [z0-R,  z0+TZ+R)   cols [x0-4, x0+124)  (128 wide)
//   sVX  x-velocity   rows [z0-R,  z0+TZ+R)   cols [x0-8, x0+128)  (136 wide)
//   sVZ  z-velocity   rows [z0-2R, z0+TZ+2R)  cols [x0-4, x0+124)  (128 wide)
//
// The p-stage updates pressure on the whole sP rectangle (tile + R-row and
// 4-column halo) in place; the v-stage then updates vx, vz on the tile from
// that halo.  The 128-wide rectangles are exactly 32 lanes x 4 columns.
// ---------------------------------------------------------------------------
constexpr int TX = 120;
constexpr int RW = 128;          // sP / sVZ row pitch (floats)
constexpr int VXW = 136;         // sVX row pitch (floats)
constexpr int NWARP = 8;
constexpr int NTHR = NWARP * 32;
constexpr int kMaxShotsPerCta = 64;

template <int R, int TZ>
struct Geo {
    static constexpr int PR = TZ + 2 * R;        // rows of sP and sVX
    static constexpr int ZR = TZ + 4 * R;        // rows of sVZ
    static constexpr int P_FL = PR * RW;
    static constexpr int VX_FL = PR * VXW;
    static constexpr int VZ_FL = ZR * RW;
    static constexpr int STAGE_FL = P_FL + VX_FL + VZ_FL;
    static constexpr uint32_t STAGE_BYTES = STAGE_FL * 4u;
    static constexpr int LP = (PR + NWARP - 1) / NWARP;   // p-stage rows per warp
    static constexpr int LV = (TZ + NWARP - 1) / NWARP;   // v-stage rows per warp
    static_assert((P_FL * 4) % 128 == 0 && (VX_FL * 4) % 128 == 0 && (VZ_FL * 4) % 128 == 0,
                  "TMA destinations must stay 128-byte aligned");
};

// Bounded waits: a wait that does not complete within this many polls (with a
// nanosleep back-off, well over a second) records GB_E_TIMEOUT and returns.
constexpr uint32_t kMaxPolls = 1u << 22;

// ---------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Programmatic dependent launch.  A step kernel launched with programmatic
// stream serialisation may start while the previous kernel of its stream is
// still running: it sets up shared memory, then waits here before it reads
// or writes anything a previous kernel touches (a no-op for a kernel
// launched without the attribute), then lets the next one launch.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Returns false (and the caller reports GB_E_TIMEOUT) if the phase never
// completes.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t max_polls = kMaxPolls)
{
    for (uint32_t i = 0; i < max_polls; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (i > 64) __nanosleep(256);
    }
    return false;
}

// 3-D tiled TMA load: box at (x, y, z) of `map` into shared memory, completion
// counted on `bar`.  x must be a multiple of 4 (16 bytes of fp32); y, z may
// be out of range (zero fill).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y,
                                            int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ float4 lds4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void sts4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float4 ldg4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ void stg4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float4 zero4() { return make_float4(0.f, 0.f, 0.f, 0.f); }

__device__ __forceinline__ float &at(float4 &v, int q)
{
    return reinterpret_cast<float *>(&v)[q];
}
__device__ __forceinline__ float at(const float4 &v, int q)
{
    return reinterpret_cast<const float *>(&v)[q];
}

// Storage formats of the imaging fields kept for the adjoint (the values of
// GB_IMG_* in the C header):
//   kImgF32   fp32;
//   kImgBF16  bf16, the upper 16 bits of the fp32 rounded to nearest even;
//   kImgF24   the upper 24 bits of the fp32 (sign, 8-bit exponent, 15-bit
//             mantissa) rounded to nearest even, 3 bytes, packed 4 values to
//             3 words.
// Both short formats keep the fp32 exponent, so no scale is needed and
// widening back is exact.  `o` is an element offset, a multiple of 4.
constexpr int kImgF32 = 0;
constexpr int kImgBF16 = 1;
constexpr int kImgF24 = 3;

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi)
{
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
// fp32 -> upper 24 bits, round to nearest even on the 8 dropped bits (a carry
// into the exponent is the correct rounding up to the next binade).
__device__ __forceinline__ uint32_t round24(float x)
{
    const uint32_t u = __float_as_uint(x);
    return (u + 0x7fu + ((u >> 8) & 1u)) >> 8;
}
__device__ __forceinline__ void store_img4(float *base, long long o, int fmt, float4 v)
{
    if (fmt == kImgBF16) {
        uint2 u = make_uint2(pack_bf16x2(v.x, v.y), pack_bf16x2(v.z, v.w));
        *reinterpret_cast<uint2 *>(reinterpret_cast<uint16_t *>(base) + o) = u;
    } else if (fmt == kImgF24) {
        const uint32_t t0 = round24(v.x), t1 = round24(v.y), t2 = round24(v.z), t3 = round24(v.w);
        uint32_t *w = reinterpret_cast<uint32_t *>(reinterpret_cast<char *>(base) + 3 * o);
        w[0] = t0 | (t1 << 24);
        w[1] = (t1 >> 8) | (t2 << 16);
        w[2] = (t2 >> 16) | (t3 << 8);
    } else {
        stg4(base + o, v);
    }
}
// Imaging values as loaded: 4 fp32 words, 2 bf16x2 words or 3 packed fp24
// words.  Loading and widening are separate so that the loads can be issued
// well ahead of the use without the widening waiting on them.
struct ImgRaw {
    uint32_t w0, w1, w2, w3;
};
__device__ __forceinline__ ImgRaw img_raw_zero() { return ImgRaw{0u, 0u, 0u, 0u}; }
__device__ __forceinline__ ImgRaw load_img_raw(const float *base, long long o, int fmt)
{
    if (fmt == kImgBF16) {
        const uint2 u = __ldg(reinterpret_cast<const uint2 *>(reinterpret_cast<const uint16_t *>(base) + o));
        return ImgRaw{u.x, u.y, 0u, 0u};
    }
    if (fmt == kImgF24) {
        const uint32_t *w = reinterpret_cast<const uint32_t *>(reinterpret_cast<const char *>(base) + 3 * o);
        return ImgRaw{__ldg(w), __ldg(w + 1), __ldg(w + 2), 0u};
    }
    const uint4 u = __ldg(reinterpret_cast<const uint4 *>(base + o));
    return ImgRaw{u.x, u.y, u.z, u.w};
}
// All-zero words widen to 0.0 in every format.
__device__ __forceinline__ float4 decode_img4(const ImgRaw &r, int fmt)
{
    if (fmt == kImgBF16)
        return make_float4(__uint_as_float(r.w0 << 16), __uint_as_float(r.w0 & 0xffff0000u),
                           __uint_as_float(r.w1 << 16), __uint_as_float(r.w1 & 0xffff0000u));
    if (fmt == kImgF24)
        return make_float4(__uint_as_float(r.w0 << 8), __uint_as_float(((r.w0 >> 24) | (r.w1 << 8)) << 8),
                           __uint_as_float(((r.w1 >> 16) | (r.w2 << 16)) << 8), __uint_as_float(r.w2 & 0xffffff00u));
    return make_float4(__uint_as_float(r.w0), __uint_as_float(r.w1), __uint_as_float(r.w2), __uint_as_float(r.w3));
}

__device__ __forceinline__ void red_add_v4(float *p, float4 v)
{
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z),
                 "f"(v.w)
                 : "memory");
}

}  // namespace gb
