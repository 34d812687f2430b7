// Small kernels around the fused step: coefficient planes (pad_model +
// coefficient preparation), energy-map extraction, snapshot packing, and the
// final gradient reduction.
#pragma once

#include "gb_device.cuh"
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace gb {

// Padded coefficient planes, Nz x pitch (columns >= Nx are zero).
// geobrain/physics/wave/kernels/acoustic_2d.py: pad_model :18-66 (index
// clamping = edge replication), alpha1/kappa1/alpha2/kappa2/kappa3 :406-420,
// in the reference's fp32 operation order.
__global__ void coef_kernel(const float *__restrict__ vp, const float *__restrict__ rho,
                            const float *__restrict__ damp, int nz, int nx, int pml, int Nz, int Nx, int pitch,
                            int fs, float dt, float dz, float *a1, float *k1, float *a2, float *k2, float *k3)
{
    const long long n = (long long)Nz * pitch;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / pitch), j = (int)(idx % pitch);
        if (j >= Nx) {
            a1[idx] = 0.f; k1[idx] = 0.f; a2[idx] = 0.f; k2[idx] = 0.f; k3[idx] = 0.f;
            continue;
        }
        const int iz = min(max(i - pml, 0), nz - 1), ix = min(max(j - pml, 0), nx - 1);
        const float c = vp[(long long)iz * nx + ix];
        const float den = rho[(long long)iz * nx + ix];
        const float d = damp[(long long)i * Nx + j];
        a1[idx] = __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(den, c), c), dt), dz);
        a2[idx] = __fdiv_rn(dt, __fmul_rn(den, dz));
        k1[idx] = __fmul_rn(d, dt);
        k2[idx] = (j >= 1 && j <= Nx - 3)
                      ? __fmul_rn(__fmul_rn(0.5f, __fadd_rn(d, damp[(long long)i * Nx + j + 1])), dt)
                      : 0.f;
        k3[idx] = (i >= fs && i <= Nz - 3)
                      ? __fmul_rn(__fmul_rn(0.5f, __fadd_rn(d, damp[(long long)(i + 1) * Nx + j])), dt)
                      : 0.f;
    }
}

// Interior (nz, nx) of a padded Nz x pitch plane.
__global__ void extract_interior_kernel(const float *__restrict__ src, int nz, int nx, int pml, int pitch,
                                        float *__restrict__ dst)
{
    const long long n = (long long)nz * nx;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int iz = (int)(idx / nx), ix = (int)(idx % nx);
        dst[idx] = src[(long long)(iz + pml) * pitch + ix + pml];
    }
}

}  // namespace gb

namespace gb {

// ---------------------------------------------------------------------------
// Checkpoint snapshots in 16 bits with one fp32 scale per (checkpoint, shot,
// field) plane.  Pass 1 takes |x|max of each plane; pass 2 stores x / scale
// (scale = absmax / 2^15, so every plane spans about +-32768, well inside the
// range of either format); unpacking multiplies back.  bf16 keeps 8
// significant bits, fp16 11; the recompute that restarts from a snapshot runs
// in fp32.
// ---------------------------------------------------------------------------
__global__ void plane_absmax_kernel(const float *__restrict__ x, long long plane, unsigned int *amax_bits)
{
    const int pl = blockIdx.y;
    const float *p = x + pl * plane;
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
         i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(p[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&amax_bits[pl], __float_as_uint(m));   // |x| >= 0 orders as unsigned
}

template <class H>
__device__ __forceinline__ H to_h(float v);
template <>
__device__ __forceinline__ __nv_bfloat16 to_h<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <>
__device__ __forceinline__ __half to_h<__half>(float v) { return __float2half_rn(v); }
__device__ __forceinline__ float from_h(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float from_h(__half v) { return __half2float(v); }

constexpr float kSnapshotRange = 32768.f;

template <class H>
__global__ void pack16_kernel(const float *__restrict__ x, long long plane, const unsigned int *__restrict__ amax_bits,
                              H *__restrict__ out, float *__restrict__ scales)
{
    const int pl = blockIdx.y;
    const float amax = __uint_as_float(amax_bits[pl]);
    // the floor keeps all-zero and subnormal-only planes finite
    const float scale = fmaxf(amax / kSnapshotRange, 1.17549435e-38f);
    const float inv = 1.f / scale;
    if (blockIdx.x == 0 && threadIdx.x == 0) scales[pl] = scale;
    const float *p = x + pl * plane;
    H *o = out + pl * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
         i += (long long)gridDim.x * blockDim.x)
        o[i] = to_h<H>(p[i] * inv);
}

template <class H>
__global__ void unpack16_kernel(const H *__restrict__ in, const float *__restrict__ scales, long long plane,
                                float *__restrict__ x)
{
    const int pl = blockIdx.y;
    const float scale = scales[pl];
    const H *p = in + pl * plane;
    float *o = x + pl * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
         i += (long long)gridDim.x * blockDim.x)
        o[i] = from_h(p[i]) * scale;
}

// Checkpoint snapshots in 24 bits: the upper 24 bits of each fp32 (sign,
// exponent, 15-bit mantissa) rounded to nearest even, 4 values to 3 words,
// the same packing as the fp24 imaging fields.  The exponent is kept, so no
// scale is needed; the relative error of each value is at most 2^-16.
__global__ void pack24_kernel(const float *__restrict__ x, long long n4, float *__restrict__ out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4;
         i += (long long)gridDim.x * blockDim.x)
        store_img4(out, 4 * i, kImgF24, ldg4(x + 4 * i));
}

__global__ void unpack24_kernel(const float *__restrict__ in, long long n4, float *__restrict__ x)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4;
         i += (long long)gridDim.x * blockDim.x)
        stg4(x + 4 * i, decode_img4(load_img_raw(in, 4 * i, kImgF24), kImgF24));
}

// Self-test of the bounded waits.  One CTA waits on an mbarrier of arrival
// count 2.  The second arrival is made only when `complete` is set, so
// otherwise the phase never completes: the wait gives up after max_polls
// polls and the CTA sets the status word to the timeout code, as every step
// kernel does when its TMA loads never land.  Nothing is in flight when it
// returns.
__global__ void bounded_wait_selftest_kernel(int *err, int complete, uint32_t max_polls)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 2);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_arrive(&bar);
        if (complete) mbar_arrive(&bar);
    }
    __syncthreads();
    if (!__syncthreads_and(mbar_wait_bounded(&bar, 0, max_polls)) && threadIdx.x == 0) atomicExch(err, -4);
}

// Step counter of graph-replayed forward chunks.
__global__ void step_set_kernel(int *ctr, int value) { *ctr = value; }
__global__ void step_advance_kernel(int *ctr, int by) { *ctr += by; }

}  // namespace gb
