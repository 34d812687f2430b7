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
