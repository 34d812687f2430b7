// 3-D acoustic staggered-grid step, 4th order
// (geobrain/physics/wave/kernels/acoustic_3d.py:20-300, driver :303-476).
//
// Per time step, for every shot:
//   p  <- (1 - k1) p - a1 (dvx/dx + dvy/dy + dvz/dz)        (ref :117-150)
//         on z [fs+1, Nz-2), y [2, Ny-2), x [2, Nx-2)
//   p[sz, sy, sx] += dt * w[s, it]                            (ref :153-163)
//   p[fs-1] = -p[fs+1]          free surface                  (ref :166-167)
//   vx <- (1 - k2) vx - a2 dp/dx   z [fs, Nz-1), y [1, Ny-1), x [1, Nx-2)
//   vy <- (1 - k3) vy - a2 dp/dy   z [fs, Nz-1), y [1, Ny-2), x [1, Nx-1)
//   vz <- (1 - k4) vz - a2 dp/dz   z [fs, Nz-2), y [1, Ny-1), x [1, Nx-1)
//                                                              (ref :170-233)
//   vz[fs-1] = vz[fs]                                          (ref :236-237)
//   traces[s, it, r] = (p, vx, vy, vz)[receiver r]             (ref :240-243)
//   energy += sum_s (p^2, vx^2, vy^2, vz^2) on the interior    (ref :246-258)
// with d/dq f = c1 (f[q] - f[q-1]) + c2 (f[q+1] - f[q-2]) at the staggered
// points, c1 = 9/8, c2 = -1/24, every operation rounded separately in the
// reference's order.
//
// Layout: [shot][p | vx | vy | vz][Nz][Ny][pitch] fp32 with pitch =
// roundup(Nx, 32); vx's last column, vy's last row and vz's last plane
// (absent in the reference) stay zero.  A thread owns 4 adjacent x cells
// of one (z, y) row and loops over the shots, so the coefficients are read
// once per step and the energy sums need no atomics.  Each update reads
// only the other fields and writes only its own, so both run in place.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gb {

struct Geo3 {
    int Nz, Ny, Nx, pitch;
    int nz, ny, nx, pml, fs;
    int n_shots, nt, n_rcv;
    float dt;
    long long plane;   // Ny * pitch
    long long vol;     // Nz * plane
};

// The shot loops below ask L2 for the next shot's cells of this thread while
// the current shot computes.  At 16-24 resident warps per SM the loads of one
// shot alone leave DRAM idle between shots; with the prefetch the 200^3,
// 4-shot forward runs 1.27x faster (the arithmetic is unchanged).  Every
// prefetched address is inside the state / imaging arrays.
__device__ __forceinline__ void prefetch_l2(const float *p)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

constexpr float kC1 = 9.0f / 8.0f;
constexpr float kC2 = -1.0f / 24.0f;

__device__ __forceinline__ float4 ld4z(const float *base, long long o, bool ok)
{
    return ok ? *reinterpret_cast<const float4 *>(base + o) : make_float4(0.f, 0.f, 0.f, 0.f);
}
__device__ __forceinline__ float f4(const float4 &v, int q)
{
    return q == 0 ? v.x : q == 1 ? v.y : q == 2 ? v.z : v.w;
}
// c1 (a - b) + c2 (c - d), rounded as the reference evaluates it
__device__ __forceinline__ float d4(float a, float b, float c, float d)
{
    return __fadd_rn(__fmul_rn(kC1, __fsub_rn(a, b)), __fmul_rn(kC2, __fsub_rn(c, d)));
}

// Coefficients from the unpadded vp / rho (edge-replicated padding as
// pad_model_3d, kernels/acoustic_2d.py:70-120) and the padded damping, in the
// reference's fp32 operation order (acoustic_3d.py:410-441).
__global__ void coef3_kernel(const Geo3 g, const float *__restrict__ vp, const float *__restrict__ rho,
                             const float *__restrict__ damp, float dz, float *a1, float *k1, float *a2, float *k2,
                             float *k3, float *k4)
{
    const long long n = (long long)g.Nz * g.Ny * g.Nx;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % g.Nx), y = (int)((i / g.Nx) % g.Ny), z = (int)(i / ((long long)g.Nx * g.Ny));
        const int zi = min(max(z - g.pml, 0), g.nz - 1), yi = min(max(y - g.pml, 0), g.ny - 1),
                  xi = min(max(x - g.pml, 0), g.nx - 1);
        const long long m = ((long long)zi * g.ny + yi) * g.nx + xi;
        const float c = vp[m], den = rho[m];
        const long long d = ((long long)z * g.Ny + y) * g.Nx + x;
        const long long o = (long long)z * g.plane + (long long)y * g.pitch + x;
        a1[o] = __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(den, c), c), g.dt), dz);
        k1[o] = __fmul_rn(damp[d], g.dt);
        a2[o] = __fdiv_rn(g.dt, __fmul_rn(den, dz));
        k2[o] = (x >= 1 && x < g.Nx - 2) ? __fmul_rn(__fmul_rn(0.5f, __fadd_rn(damp[d], damp[d + 1])), g.dt) : 0.f;
        k3[o] = (y >= 1 && y < g.Ny - 2) ? __fmul_rn(__fmul_rn(0.5f, __fadd_rn(damp[d], damp[d + g.Nx])), g.dt)
                                         : 0.f;
        k4[o] = (z >= g.fs && z < g.Nz - 2)
                    ? __fmul_rn(__fmul_rn(0.5f, __fadd_rn(damp[d], damp[d + (long long)g.Nx * g.Ny])), g.dt)
                    : 0.f;
    }
}

struct Args3 {
    Geo3 g;
    int it;
    const int *step_base;                 // device step counter (graph replay) or null
    float *state;                         // [S][4][Nz][Ny][pitch]
    const float *a1, *k1, *a2, *k2, *k3, *k4;
    const int *src;                       // [3][S]: padded z, y, x
    const float *wavelet;                 // [S][nt]
    float *energy[4];                     // (nz, ny, nx) accumulators or null
    float *img_i;                         // gradient recompute: -(dvx+dvy+dvz) per p cell [S][vol], or null
    float *img_j;                         // and dp/dx, dp/dy, dp/dz per v cell [3][S][vol] (density), or null
};

__device__ __forceinline__ int step_of(const Args3 &A)
{
    return A.step_base ? *reinterpret_cast<const volatile int *>(A.step_base) + A.it : A.it;
}

// p update and source (block: 32 x-quads x 4 rows; grid: x-blocks, y-blocks, Nz).
// The register bounds of the four step kernels (8, 7, 4, 4 CTAs per SM) trade
// a few spilled bytes for resident warps; measured at 200^3 with 4 shots,
// the forward runs 7 % faster than at the compiler's own choice.
__global__ void __launch_bounds__(128, 8) p3_kernel(const Args3 A)
{
    const Geo3 &g = A.g;
    const int x0 = 4 * (blockIdx.x * 32 + threadIdx.x);
    const int y = blockIdx.y * 4 + threadIdx.y;
    const int z = blockIdx.z;
    if (x0 >= g.Nx || y >= g.Ny) return;
    const int it = step_of(A);
    const long long o = (long long)z * g.plane + (long long)y * g.pitch + x0;
    const bool row_in = z >= g.fs + 1 && z < g.Nz - 2 && y >= 2 && y < g.Ny - 2 && x0 + 3 >= 2 && x0 < g.Nx - 2;
    float4 a1 = make_float4(0.f, 0.f, 0.f, 0.f), k1 = a1;
    if (row_in) {
        a1 = *reinterpret_cast<const float4 *>(A.a1 + o);
        k1 = *reinterpret_cast<const float4 *>(A.k1 + o);
    }
    // the p energy is complete once p is: the free-surface mirror plane
    // (fs - 1 = pml - 1) lies outside the interior
    const bool energy = A.energy[0] && z >= g.pml && z < g.pml + g.nz && y >= g.pml && y < g.pml + g.ny;
    float e[4] = {0.f, 0.f, 0.f, 0.f};
    for (int s = 0; s < g.n_shots; ++s) {
        float *P = A.state + (long long)s * 4 * g.vol;
        const float *VX = P + g.vol, *VY = P + 2 * g.vol, *VZ = P + 3 * g.vol;
        if (s + 1 < g.n_shots) {
            const float *N = P + 4 * g.vol + o;
            prefetch_l2(N); prefetch_l2(N + g.vol); prefetch_l2(N + 2 * g.vol); prefetch_l2(N + 3 * g.vol);
        }
        float4 p = *reinterpret_cast<const float4 *>(P + o);
        if (row_in) {
            const float4 xl = ld4z(VX, o - 4, x0 >= 4), xc = ld4z(VX, o, true),
                         xr = ld4z(VX, o + 4, x0 + 4 < g.pitch);
            const float xs[12] = {xl.x, xl.y, xl.z, xl.w, xc.x, xc.y, xc.z, xc.w, xr.x, xr.y, xr.z, xr.w};
            const float4 ym2 = ld4z(VY, o - 2 * g.pitch, true), ym1 = ld4z(VY, o - g.pitch, true),
                         y0 = ld4z(VY, o, true), yp1 = ld4z(VY, o + g.pitch, true);
            const float4 zm2 = ld4z(VZ, o - 2 * g.plane, true), zm1 = ld4z(VZ, o - g.plane, true),
                         z0 = ld4z(VZ, o, true), zp1 = ld4z(VZ, o + g.plane, true);
            float pv[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int x = x0 + q;
                if (x < 2 || x >= g.Nx - 2) continue;
                const float dvx = d4(xs[q + 4], xs[q + 3], xs[q + 5], xs[q + 2]);
                const float dvy = d4(f4(y0, q), f4(ym1, q), f4(yp1, q), f4(ym2, q));
                const float dvz = d4(f4(z0, q), f4(zm1, q), f4(zp1, q), f4(zm2, q));
                const float sum = __fadd_rn(__fadd_rn(dvx, dvy), dvz);
                pv[q] = __fsub_rn(__fmul_rn(__fsub_rn(1.f, f4(k1, q)), pv[q]), __fmul_rn(f4(a1, q), sum));
                if (A.img_i) A.img_i[(long long)s * g.vol + o + q] = -sum;
            }
            p = make_float4(pv[0], pv[1], pv[2], pv[3]);
        }
        const int sz = A.src[s], sy = A.src[g.n_shots + s], sx = A.src[2 * g.n_shots + s];
        if (sz == z && sy == y && sx >= x0 && sx < x0 + 4) {
            const float amp = __fmul_rn(g.dt, A.wavelet[(long long)s * g.nt + it]);
            const int q = sx - x0;
            if (q == 0) p.x = __fadd_rn(p.x, amp);
            else if (q == 1) p.y = __fadd_rn(p.y, amp);
            else if (q == 2) p.z = __fadd_rn(p.z, amp);
            else p.w = __fadd_rn(p.w, amp);
        }
        *reinterpret_cast<float4 *>(P + o) = p;
        if (energy) {
#pragma unroll
            for (int q = 0; q < 4; ++q) e[q] = __fadd_rn(e[q], __fmul_rn(f4(p, q), f4(p, q)));
        }
    }
    if (energy) {
        const long long eo = ((long long)(z - g.pml) * g.ny + (y - g.pml)) * g.nx - g.pml;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int x = x0 + q;
            if (x >= g.pml && x < g.pml + g.nx) A.energy[0][eo + x] = __fadd_rn(A.energy[0][eo + x], e[q]);
        }
    }
}

// Free-surface mirror plane of field f: f[fs-1] = sign * f[fs - 1 + from]
__global__ void mirror3_kernel(const Geo3 g, float *state, int field, int from, float sign)
{
    const long long n = (long long)g.n_shots * g.plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long s = i / g.plane, r = i % g.plane;
        float *F = state + (s * 4 + field) * g.vol;
        F[(long long)(g.fs - 1) * g.plane + r] = sign * F[(long long)(g.fs - 1 + from) * g.plane + r];
    }
}

// vx, vy, vz updates and their energy sums (same blocks as p3_kernel)
__global__ void __launch_bounds__(128, 7) v3_kernel(const Args3 A)
{
    const Geo3 &g = A.g;
    const int x0 = 4 * (blockIdx.x * 32 + threadIdx.x);
    const int y = blockIdx.y * 4 + threadIdx.y;
    const int z = blockIdx.z;
    if (x0 >= g.Nx || y >= g.Ny) return;
    const long long o = (long long)z * g.plane + (long long)y * g.pitch + x0;
    const bool zin = z >= g.fs && z < g.Nz - 1;
    const bool vx_row = zin && y >= 1 && y < g.Ny - 1;
    const bool vy_row = zin && y >= 1 && y < g.Ny - 2;
    const bool vz_row = z >= g.fs && z < g.Nz - 2 && y >= 1 && y < g.Ny - 1;
    const bool any = vx_row || vy_row || vz_row;
    float4 a2 = make_float4(0.f, 0.f, 0.f, 0.f), k2 = a2, k3 = a2, k4 = a2;
    if (any) {
        a2 = *reinterpret_cast<const float4 *>(A.a2 + o);
        k2 = *reinterpret_cast<const float4 *>(A.k2 + o);
        k3 = *reinterpret_cast<const float4 *>(A.k3 + o);
        k4 = *reinterpret_cast<const float4 *>(A.k4 + o);
    }
    const bool interior_row = z >= g.pml && z < g.pml + g.nz && y >= g.pml && y < g.pml + g.ny;
    const bool energy = interior_row && A.energy[0];
    float e[3][4] = {};
    for (int s = 0; s < g.n_shots; ++s) {
        float *P = A.state + (long long)s * 4 * g.vol;
        float *VX = P + g.vol, *VY = P + 2 * g.vol, *VZ = P + 3 * g.vol;
        if (s + 1 < g.n_shots) {
            const float *N = P + 4 * g.vol + o;
            prefetch_l2(N); prefetch_l2(N + g.vol); prefetch_l2(N + 2 * g.vol); prefetch_l2(N + 3 * g.vol);
        }
        const float4 pc = *reinterpret_cast<const float4 *>(P + o);
        float4 vx = *reinterpret_cast<const float4 *>(VX + o);
        float4 vy = *reinterpret_cast<const float4 *>(VY + o);
        float4 vz = *reinterpret_cast<const float4 *>(VZ + o);
        if (any) {
            const float4 pl = ld4z(P, o - 4, x0 >= 4), pr = ld4z(P, o + 4, x0 + 4 < g.pitch);
            const float ps[12] = {pl.x, pl.y, pl.z, pl.w, pc.x, pc.y, pc.z, pc.w, pr.x, pr.y, pr.z, pr.w};
            float rx[4] = {vx.x, vx.y, vx.z, vx.w}, ry[4] = {vy.x, vy.y, vy.z, vy.w}, rz[4] = {vz.x, vz.y, vz.z, vz.w};
            if (vx_row) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int x = x0 + q;
                    if (x < 1 || x >= g.Nx - 2) continue;
                    const float dp = d4(ps[q + 5], ps[q + 4], ps[q + 6], ps[q + 3]);
                    rx[q] = __fsub_rn(__fmul_rn(__fsub_rn(1.f, f4(k2, q)), rx[q]), __fmul_rn(f4(a2, q), dp));
                    if (A.img_j) A.img_j[(long long)s * g.vol + o + q] = dp;
                }
            }
            if (vy_row) {
                const float4 ym1 = ld4z(P, o - g.pitch, true), yp1 = ld4z(P, o + g.pitch, true),
                             yp2 = ld4z(P, o + 2 * g.pitch, true);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int x = x0 + q;
                    if (x < 1 || x >= g.Nx - 1) continue;
                    const float dp = d4(f4(yp1, q), f4(pc, q), f4(yp2, q), f4(ym1, q));
                    ry[q] = __fsub_rn(__fmul_rn(__fsub_rn(1.f, f4(k3, q)), ry[q]), __fmul_rn(f4(a2, q), dp));
                    if (A.img_j) A.img_j[((long long)g.n_shots + s) * g.vol + o + q] = dp;
                }
            }
            if (vz_row) {
                const float4 zm1 = ld4z(P, o - g.plane, true), zp1 = ld4z(P, o + g.plane, true),
                             zp2 = ld4z(P, o + 2 * g.plane, true);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int x = x0 + q;
                    if (x < 1 || x >= g.Nx - 1) continue;
                    const float dp = d4(f4(zp1, q), f4(pc, q), f4(zp2, q), f4(zm1, q));
                    rz[q] = __fsub_rn(__fmul_rn(__fsub_rn(1.f, f4(k4, q)), rz[q]), __fmul_rn(f4(a2, q), dp));
                    if (A.img_j) A.img_j[(2LL * g.n_shots + s) * g.vol + o + q] = dp;
                }
            }
            vx = make_float4(rx[0], rx[1], rx[2], rx[3]);
            vy = make_float4(ry[0], ry[1], ry[2], ry[3]);
            vz = make_float4(rz[0], rz[1], rz[2], rz[3]);
            *reinterpret_cast<float4 *>(VX + o) = vx;
            *reinterpret_cast<float4 *>(VY + o) = vy;
            *reinterpret_cast<float4 *>(VZ + o) = vz;
        }
        if (energy) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                e[0][q] = __fadd_rn(e[0][q], __fmul_rn(f4(vx, q), f4(vx, q)));
                e[1][q] = __fadd_rn(e[1][q], __fmul_rn(f4(vy, q), f4(vy, q)));
                e[2][q] = __fadd_rn(e[2][q], __fmul_rn(f4(vz, q), f4(vz, q)));
            }
        }
    }
    if (energy) {
        // this thread is the only writer of these cells
        const long long eo = ((long long)(z - g.pml) * g.ny + (y - g.pml)) * g.nx;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int x = x0 + q;
            if (x < g.pml || x >= g.pml + g.nx) continue;
            for (int f = 0; f < 3; ++f)
                A.energy[f + 1][eo + x - g.pml] = __fadd_rn(A.energy[f + 1][eo + x - g.pml], e[f][q]);
        }
    }
}

// Receivers: traces[f][s][it][r] = field f at the receiver (padded z, y, x)
__global__ void rec3_kernel(const Geo3 g, const float *state, const int *rcv, float *tr_p, float *tr_vx,
                            float *tr_vy, float *tr_vz, int it, const int *step_base)
{
    const long long n = (long long)g.n_shots * g.n_rcv;
    if (step_base) it += *reinterpret_cast<const volatile int *>(step_base);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / g.n_rcv), r = (int)(i % g.n_rcv);
        const long long o = (long long)rcv[r] * g.plane + (long long)rcv[g.n_rcv + r] * g.pitch + rcv[2 * g.n_rcv + r];
        const float *P = state + (long long)s * 4 * g.vol;
        const long long t = ((long long)s * g.nt + it) * g.n_rcv + r;
        if (tr_p) tr_p[t] = P[o];
        if (tr_vx) tr_vx[t] = P[g.vol + o];
        if (tr_vy) tr_vy[t] = P[2 * g.vol + o];
        if (tr_vz) tr_vz[t] = P[3 * g.vol + o];
    }
}

// ---------------------------------------------------------------------------
// Adjoint (reverse time) of one step, in gather form.  lam = adjoint of the
// state after the step; the two kernels below undo the velocity updates and
// then the pressure update:
//   adj_v3: lp' = lp + sum_c -G_c^T (a2 lam_c on M_c),  lam_c' = (1 - k_c) lam_c on M_c
//   adj_p3: lp  = (1 - k1) lp' on M_p,  lam_c = lam_c' - D_c^T (a1 lp' on M_p)
// with (G^T w)[q] = c1 (w[q-1] - w[q]) + c2 (w[q-2] - w[q+1]) and
// (D^T u)[q] = c1 (u[q] - u[q+1]) + c2 (u[q-1] - u[q+2]) along each
// component's axis, and the gradient sums dL/da1 += lp' I, dL/da2 +=
// -lam_c J_c (Neumaier-compensated, one owner per cell, no atomics).
// ---------------------------------------------------------------------------
struct AdjArgs3 {
    Geo3 g;
    const float *lam_in;          // [S][4][vol] adjoint state
    float *lam_out;
    const float *a1, *k1, *a2, *k2, *k3, *k4;
    const float *img_i, *img_j;   // this step's recomputed imaging fields
    float *G1, *C1, *G2, *C2;     // [vol] gradient sums and compensations (G2 / C2 null without density)
};

__device__ __forceinline__ void neumaier3(float &s, float &c, float x)
{
    const float t = s + x;
    if (fabsf(s) >= fabsf(x))
        c += (s - t) + x;
    else
        c += (x - t) + s;
    s = t;
}

__device__ __forceinline__ bool in_px(const Geo3 &g, int x) { return x >= 2 && x < g.Nx - 2; }
__device__ __forceinline__ bool in_p(const Geo3 &g, int z, int y, int x)
{
    return z >= g.fs + 1 && z < g.Nz - 2 && y >= 2 && y < g.Ny - 2 && in_px(g, x);
}
__device__ __forceinline__ bool in_vx(const Geo3 &g, int z, int y, int x)
{
    return z >= g.fs && z < g.Nz - 1 && y >= 1 && y < g.Ny - 1 && x >= 1 && x < g.Nx - 2;
}
__device__ __forceinline__ bool in_vy(const Geo3 &g, int z, int y, int x)
{
    return z >= g.fs && z < g.Nz - 1 && y >= 1 && y < g.Ny - 2 && x >= 1 && x < g.Nx - 1;
}
__device__ __forceinline__ bool in_vz(const Geo3 &g, int z, int y, int x)
{
    return z >= g.fs && z < g.Nz - 2 && y >= 1 && y < g.Ny - 1 && x >= 1 && x < g.Nx - 1;
}
// value at (z, y, x) of field f, 0 outside the grid
__device__ __forceinline__ float at3(const Geo3 &g, const float *F, int z, int y, int x)
{
    if (z < 0 || z >= g.Nz || y < 0 || y >= g.Ny || x < 0 || x >= g.Nx) return 0.f;
    return F[(long long)z * g.plane + (long long)y * g.pitch + x];
}

// float4 of field F at (z, y, x4), 0 outside the grid rows / planes; x4 is a
// multiple of 4 and x4 - 4 >= 0 is checked by the caller's guard
__device__ __forceinline__ float4 row4(const Geo3 &g, const float *F, int z, int y, int x4)
{
    if (z < 0 || z >= g.Nz || y < 0 || y >= g.Ny || x4 < 0 || x4 >= g.pitch) return make_float4(0.f, 0.f, 0.f, 0.f);
    return *reinterpret_cast<const float4 *>(F + (long long)z * g.plane + (long long)y * g.pitch + x4);
}

__global__ void __launch_bounds__(128, 4) adj_v3_kernel(const AdjArgs3 A)
{
    const Geo3 &g = A.g;
    const int x0 = 4 * (blockIdx.x * 32 + threadIdx.x);
    const int y = blockIdx.y * 4 + threadIdx.y;
    const int z = blockIdx.z;
    if (x0 >= g.Nx || y >= g.Ny) return;
    const long long o = (long long)z * g.plane + (long long)y * g.pitch + x0;
    // a2 times the mask of each velocity component at the neighbours the
    // transposed gradient reads: x-1 .. x+1 (vx), rows y-2 .. y+1 (vy),
    // planes z-2 .. z+1 (vz); the same for every shot
    float mx[12], my[4][4], mz[4][4];
    {
        const float4 l = row4(g, A.a2, z, y, x0 - 4), c = row4(g, A.a2, z, y, x0), r = row4(g, A.a2, z, y, x0 + 4);
        const float v[12] = {l.x, l.y, l.z, l.w, c.x, c.y, c.z, c.w, r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 12; ++i) mx[i] = in_vx(g, z, y, x0 - 4 + i) ? v[i] : 0.f;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float4 ay = row4(g, A.a2, z, y + k - 2, x0), az = row4(g, A.a2, z + k - 2, y, x0);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            my[k][q] = in_vy(g, z, y + k - 2, x0 + q) ? f4(ay, q) : 0.f;
            mz[k][q] = in_vz(g, z + k - 2, y, x0 + q) ? f4(az, q) : 0.f;
        }
    }
    const float4 k2 = row4(g, A.k2, z, y, x0), k3 = row4(g, A.k3, z, y, x0), k4 = row4(g, A.k4, z, y, x0);
    float g2[4] = {0.f, 0.f, 0.f, 0.f};
    for (int s = 0; s < g.n_shots; ++s) {
        const float *L = A.lam_in + (long long)s * 4 * g.vol;
        float *O = A.lam_out + (long long)s * 4 * g.vol;
        const float *LX = L + g.vol, *LY = L + 2 * g.vol, *LZ = L + 3 * g.vol;
        if (s + 1 < g.n_shots) {
            const float *N = L + 4 * g.vol + o;
            prefetch_l2(N); prefetch_l2(N + g.vol); prefetch_l2(N + 2 * g.vol); prefetch_l2(N + 3 * g.vol);
            if (A.G2) {
                const long long js = (long long)g.n_shots * g.vol, jo = (long long)(s + 1) * g.vol + o;
                prefetch_l2(A.img_j + jo); prefetch_l2(A.img_j + js + jo); prefetch_l2(A.img_j + 2 * js + jo);
            }
        }
        const float4 xl = row4(g, LX, z, y, x0 - 4), xc = row4(g, LX, z, y, x0), xr = row4(g, LX, z, y, x0 + 4);
        const float lxs[12] = {xl.x, xl.y, xl.z, xl.w, xc.x, xc.y, xc.z, xc.w, xr.x, xr.y, xr.z, xr.w};
        float4 ly[4], lz[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            ly[k] = row4(g, LY, z, y + k - 2, x0);
            lz[k] = row4(g, LZ, z + k - 2, y, x0);
        }
        const float4 lp = *reinterpret_cast<const float4 *>(L + o);
        float4 jx = make_float4(0.f, 0.f, 0.f, 0.f), jy = jx, jz = jx;
        if (A.G2) {
            const long long jo = (long long)s * g.vol + o, js = (long long)g.n_shots * g.vol;
            jx = *reinterpret_cast<const float4 *>(A.img_j + jo);
            jy = *reinterpret_cast<const float4 *>(A.img_j + js + jo);
            jz = *reinterpret_cast<const float4 *>(A.img_j + 2 * js + jo);
        }
        float op[4], ox[4], oy[4], oz[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            // w = a2 lam on the component's mask; lp' = lp - sum_c G_c^T w
            const float wx_m1 = mx[q + 3] * lxs[q + 3], wx_0 = mx[q + 4] * lxs[q + 4];
            const float wx_m2 = mx[q + 2] * lxs[q + 2], wx_p1 = mx[q + 5] * lxs[q + 5];
            const float wy_m2 = my[0][q] * f4(ly[0], q), wy_m1 = my[1][q] * f4(ly[1], q);
            const float wy_0 = my[2][q] * f4(ly[2], q), wy_p1 = my[3][q] * f4(ly[3], q);
            const float wz_m2 = mz[0][q] * f4(lz[0], q), wz_m1 = mz[1][q] * f4(lz[1], q);
            const float wz_0 = mz[2][q] * f4(lz[2], q), wz_p1 = mz[3][q] * f4(lz[3], q);
            const float gt = kC1 * (wx_m1 - wx_0) + kC2 * (wx_m2 - wx_p1) + kC1 * (wy_m1 - wy_0) +
                             kC2 * (wy_m2 - wy_p1) + kC1 * (wz_m1 - wz_0) + kC2 * (wz_m2 - wz_p1);
            op[q] = f4(lp, q) - gt;
            const int x = x0 + q;
            const float lxq = lxs[q + 4], lyq = f4(ly[2], q), lzq = f4(lz[2], q);
            const bool bx = in_vx(g, z, y, x), by = in_vy(g, z, y, x), bz = in_vz(g, z, y, x);
            ox[q] = bx ? (1.f - f4(k2, q)) * lxq : lxq;
            oy[q] = by ? (1.f - f4(k3, q)) * lyq : lyq;
            oz[q] = bz ? (1.f - f4(k4, q)) * lzq : lzq;
            if (A.G2) {
                if (bx) g2[q] -= lxq * f4(jx, q);
                if (by) g2[q] -= lyq * f4(jy, q);
                if (bz) g2[q] -= lzq * f4(jz, q);
            }
        }
        *reinterpret_cast<float4 *>(O + o) = make_float4(op[0], op[1], op[2], op[3]);
        *reinterpret_cast<float4 *>(O + g.vol + o) = make_float4(ox[0], ox[1], ox[2], ox[3]);
        *reinterpret_cast<float4 *>(O + 2 * g.vol + o) = make_float4(oy[0], oy[1], oy[2], oy[3]);
        *reinterpret_cast<float4 *>(O + 3 * g.vol + o) = make_float4(oz[0], oz[1], oz[2], oz[3]);
    }
    if (A.G2) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (x0 + q < g.Nx) neumaier3(A.G2[o + q], A.C2[o + q], g2[q]);
    }
}

__global__ void __launch_bounds__(128, 4) adj_p3_kernel(const AdjArgs3 A)
{
    const Geo3 &g = A.g;
    const int x0 = 4 * (blockIdx.x * 32 + threadIdx.x);
    const int y = blockIdx.y * 4 + threadIdx.y;
    const int z = blockIdx.z;
    if (x0 >= g.Nx || y >= g.Ny) return;
    const long long o = (long long)z * g.plane + (long long)y * g.pitch + x0;
    // a1 times the p mask at the neighbours the transposed divergence reads:
    // x-1 .. x+2, rows y-1 .. y+2, planes z-1 .. z+2 (the same for every shot)
    float ux[12], uy[4][4], uz[4][4];
    {
        const float4 l = row4(g, A.a1, z, y, x0 - 4), c = row4(g, A.a1, z, y, x0), r = row4(g, A.a1, z, y, x0 + 4);
        const float v[12] = {l.x, l.y, l.z, l.w, c.x, c.y, c.z, c.w, r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 12; ++i) ux[i] = in_p(g, z, y, x0 - 4 + i) ? v[i] : 0.f;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float4 ay = row4(g, A.a1, z, y + k - 1, x0), az = row4(g, A.a1, z + k - 1, y, x0);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uy[k][q] = in_p(g, z, y + k - 1, x0 + q) ? f4(ay, q) : 0.f;
            uz[k][q] = in_p(g, z + k - 1, y, x0 + q) ? f4(az, q) : 0.f;
        }
    }
    const float4 k1 = row4(g, A.k1, z, y, x0);
    float g1[4] = {0.f, 0.f, 0.f, 0.f};
    for (int s = 0; s < g.n_shots; ++s) {
        const float *L = A.lam_in + (long long)s * 4 * g.vol;     // lp' and lam_c'
        float *O = A.lam_out + (long long)s * 4 * g.vol;
        if (s + 1 < g.n_shots) {
            const float *N = L + 4 * g.vol + o;
            prefetch_l2(N); prefetch_l2(N + g.vol); prefetch_l2(N + 2 * g.vol); prefetch_l2(N + 3 * g.vol);
            prefetch_l2(A.img_i + (long long)(s + 1) * g.vol + o);
        }
        const float4 pl = row4(g, L, z, y, x0 - 4), pc = row4(g, L, z, y, x0), pr = row4(g, L, z, y, x0 + 4);
        const float ps[12] = {pl.x, pl.y, pl.z, pl.w, pc.x, pc.y, pc.z, pc.w, pr.x, pr.y, pr.z, pr.w};
        float4 py[4], pz[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            py[k] = k == 1 ? pc : row4(g, L, z, y + k - 1, x0);
            pz[k] = k == 1 ? pc : row4(g, L, z + k - 1, y, x0);
        }
        const float4 lvx = *reinterpret_cast<const float4 *>(L + g.vol + o);
        const float4 lvy = *reinterpret_cast<const float4 *>(L + 2 * g.vol + o);
        const float4 lvz = *reinterpret_cast<const float4 *>(L + 3 * g.vol + o);
        const float4 im = *reinterpret_cast<const float4 *>(A.img_i + (long long)s * g.vol + o);
        float op[4], ox[4], oy[4], oz[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int x = x0 + q;
            const float lp = ps[q + 4];
            const bool mp = in_p(g, z, y, x);
            op[q] = mp ? (1.f - f4(k1, q)) * lp : lp;
            if (mp) g1[q] += lp * f4(im, q);
            // u = a1 lp' on the p mask; lam_c = lam_c' - D_c^T u
            const float u0 = ux[q + 4] * ps[q + 4], uxp1 = ux[q + 5] * ps[q + 5];
            const float uxm1 = ux[q + 3] * ps[q + 3], uxp2 = ux[q + 6] * ps[q + 6];
            ox[q] = f4(lvx, q) - (kC1 * (u0 - uxp1) + kC2 * (uxm1 - uxp2));
            const float uym1 = uy[0][q] * f4(py[0], q), uyp1 = uy[2][q] * f4(py[2], q), uyp2 = uy[3][q] * f4(py[3], q);
            oy[q] = f4(lvy, q) - (kC1 * (u0 - uyp1) + kC2 * (uym1 - uyp2));
            const float uzm1 = uz[0][q] * f4(pz[0], q), uzp1 = uz[2][q] * f4(pz[2], q), uzp2 = uz[3][q] * f4(pz[3], q);
            oz[q] = f4(lvz, q) - (kC1 * (u0 - uzp1) + kC2 * (uzm1 - uzp2));
        }
        *reinterpret_cast<float4 *>(O + o) = make_float4(op[0], op[1], op[2], op[3]);
        *reinterpret_cast<float4 *>(O + g.vol + o) = make_float4(ox[0], ox[1], ox[2], ox[3]);
        *reinterpret_cast<float4 *>(O + 2 * g.vol + o) = make_float4(oy[0], oy[1], oy[2], oy[3]);
        *reinterpret_cast<float4 *>(O + 3 * g.vol + o) = make_float4(oz[0], oz[1], oz[2], oz[3]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
        if (x0 + q < g.Nx) neumaier3(A.G1[o + q], A.C1[o + q], g1[q]);
}

// dL/dwavelet[s, it] = dt * lam_p at the source cell, read after the adjoint
// of the velocity updates and the free-surface fold (lam_p is then the
// adjoint of p just after the source was added, acoustic_3d.py:153-163)
__global__ void wavelet_grad3_kernel(const Geo3 g, const float *lam, const int *src, float *grad_wavelet, int it)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.n_shots) return;
    const long long o = (long long)src[s] * g.plane + (long long)src[g.n_shots + s] * g.pitch + src[2 * g.n_shots + s];
    grad_wavelet[(long long)s * g.nt + it] = g.dt * lam[(long long)s * 4 * g.vol + o];
}

// Adjoint of the recording: lam[field][receiver cell] += res[field][s][it][r]
__global__ void inj3_kernel(const Geo3 g, float *lam, const int *rcv, const float *res_p, const float *res_vx,
                            const float *res_vy, const float *res_vz, int it)
{
    const long long n = (long long)g.n_shots * g.n_rcv;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / g.n_rcv), r = (int)(i % g.n_rcv);
        const long long o = (long long)rcv[r] * g.plane + (long long)rcv[g.n_rcv + r] * g.pitch + rcv[2 * g.n_rcv + r];
        float *L = lam + (long long)s * 4 * g.vol;
        const long long t = ((long long)s * g.nt + it) * g.n_rcv + r;
        if (res_p) atomicAdd(L + o, res_p[t]);     // receivers may share a cell
        if (res_vx) atomicAdd(L + g.vol + o, res_vx[t]);
        if (res_vy) atomicAdd(L + 2 * g.vol + o, res_vy[t]);
        if (res_vz) atomicAdd(L + 3 * g.vol + o, res_vz[t]);
    }
}

// Free-surface folds of the adjoint: field f, plane fs - 1 folded into plane
// fs - 1 + to with sign, then cleared (the adjoints of vz[fs-1] = vz[fs]
// and p[fs-1] = -p[fs+1]).
__global__ void fold3_kernel(const Geo3 g, float *lam, int field, int to, float sign)
{
    const long long n = (long long)g.n_shots * g.plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long s = i / g.plane, r = i % g.plane;
        float *F = lam + (s * 4 + field) * g.vol;
        F[(long long)(g.fs - 1 + to) * g.plane + r] += sign * F[(long long)(g.fs - 1) * g.plane + r];
        F[(long long)(g.fs - 1) * g.plane + r] = 0.f;
    }
}

// dL/dvp, dL/drho on the unpadded grid: the chain rule through a1 = rho c^2
// dt / dz and a2 = dt / (rho dz) on the padded grid, summed over the padded
// cells each model cell was replicated into (the adjoint of pad_model_3d).
__global__ void grad3_finish_kernel(const Geo3 g, const float *vp, const float *rho, float dz, const float *G1,
                                    const float *C1, const float *G2, const float *C2, float *grad_vp,
                                    float *grad_rho)
{
    const long long n = (long long)g.nz * g.ny * g.nx;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i % g.nx), iy = (int)((i / g.nx) % g.ny), iz = (int)(i / ((long long)g.nx * g.ny));
        const double c = vp[i], den = rho[i], dt = g.dt;
        auto range = [&](int idx, int n_in, int pml, int &lo, int &hi) {
            lo = idx == 0 ? 0 : idx + pml;
            hi = idx == n_in - 1 ? n_in + 2 * pml - 1 : idx + pml;
        };
        int z0, z1, y0, y1, x0, x1;
        range(iz, g.nz, g.pml, z0, z1);
        range(iy, g.ny, g.pml, y0, y1);
        range(ix, g.nx, g.pml, x0, x1);
        double s1 = 0.0, s2 = 0.0;
        for (int z = z0; z <= z1; ++z)
            for (int y = y0; y <= y1; ++y)
                for (int x = x0; x <= x1; ++x) {
                    const long long o = (long long)z * g.plane + (long long)y * g.pitch + x;
                    s1 += (double)G1[o] + (double)C1[o];
                    if (G2) s2 += (double)G2[o] + (double)C2[o];
                }
        grad_vp[i] = (float)(s1 * 2.0 * den * c * dt / dz);
        if (grad_rho) grad_rho[i] = (float)(s1 * c * c * dt / dz - s2 * dt / (den * den * dz));
    }
}

}  // namespace gb
