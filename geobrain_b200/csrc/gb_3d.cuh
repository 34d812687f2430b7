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

// p update and source (block: 32 x-quads x 4 rows; grid: x-blocks, y-blocks, Nz)
__global__ void __launch_bounds__(128) p3_kernel(const Args3 A)
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
    for (int s = 0; s < g.n_shots; ++s) {
        float *P = A.state + (long long)s * 4 * g.vol;
        const float *VX = P + g.vol, *VY = P + 2 * g.vol, *VZ = P + 3 * g.vol;
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

// vx, vy, vz updates and the energy sums (same blocks as p3_kernel)
__global__ void __launch_bounds__(128) v3_kernel(const Args3 A)
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
    float e[4][4] = {};
    for (int s = 0; s < g.n_shots; ++s) {
        float *P = A.state + (long long)s * 4 * g.vol;
        float *VX = P + g.vol, *VY = P + 2 * g.vol, *VZ = P + 3 * g.vol;
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
                e[0][q] = __fadd_rn(e[0][q], __fmul_rn(f4(pc, q), f4(pc, q)));
                e[1][q] = __fadd_rn(e[1][q], __fmul_rn(f4(vx, q), f4(vx, q)));
                e[2][q] = __fadd_rn(e[2][q], __fmul_rn(f4(vy, q), f4(vy, q)));
                e[3][q] = __fadd_rn(e[3][q], __fmul_rn(f4(vz, q), f4(vz, q)));
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
            for (int f = 0; f < 4; ++f) A.energy[f][eo + x - g.pml] = __fadd_rn(A.energy[f][eo + x - g.pml], e[f][q]);
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

__global__ void __launch_bounds__(128) adj_v3_kernel(const AdjArgs3 A)
{
    const Geo3 &g = A.g;
    const int x0 = 4 * (blockIdx.x * 32 + threadIdx.x);
    const int y = blockIdx.y * 4 + threadIdx.y;
    const int z = blockIdx.z;
    if (x0 >= g.Nx || y >= g.Ny) return;
    const long long o = (long long)z * g.plane + (long long)y * g.pitch + x0;
    float g2[4] = {0.f, 0.f, 0.f, 0.f};
    for (int s = 0; s < g.n_shots; ++s) {
        const float *L = A.lam_in + (long long)s * 4 * g.vol;
        float *O = A.lam_out + (long long)s * 4 * g.vol;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int x = x0 + q;
            if (x >= g.Nx) break;
            // lp' = lp - sum_c G_c^T w_c, w_c = a2 lam_c on M_c
            float acc = L[o + q];
            float gt = 0.f;
            {   // vx: w at x-1, x, x-2, x+1
                const float *W = L + g.vol;
                auto w = [&](int xx) { return in_vx(g, z, y, xx) ? at3(g, A.a2, z, y, xx) * at3(g, W, z, y, xx) : 0.f; };
                gt += kC1 * (w(x - 1) - w(x)) + kC2 * (w(x - 2) - w(x + 1));
            }
            {   // vy: rows y-1, y, y-2, y+1
                const float *W = L + 2 * g.vol;
                auto w = [&](int yy) { return in_vy(g, z, yy, x) ? at3(g, A.a2, z, yy, x) * at3(g, W, z, yy, x) : 0.f; };
                gt += kC1 * (w(y - 1) - w(y)) + kC2 * (w(y - 2) - w(y + 1));
            }
            {   // vz: planes z-1, z, z-2, z+1
                const float *W = L + 3 * g.vol;
                auto w = [&](int zz) { return in_vz(g, zz, y, x) ? at3(g, A.a2, zz, y, x) * at3(g, W, zz, y, x) : 0.f; };
                gt += kC1 * (w(z - 1) - w(z)) + kC2 * (w(z - 2) - w(z + 1));
            }
            acc -= gt;
            O[o + q] = acc;
            // own velocity cells
            const float lx = L[g.vol + o + q], ly = L[2 * g.vol + o + q], lz = L[3 * g.vol + o + q];
            const bool mx = in_vx(g, z, y, x), my = in_vy(g, z, y, x), mz = in_vz(g, z, y, x);
            O[g.vol + o + q] = mx ? (1.f - A.k2[o + q]) * lx : lx;
            O[2 * g.vol + o + q] = my ? (1.f - A.k3[o + q]) * ly : ly;
            O[3 * g.vol + o + q] = mz ? (1.f - A.k4[o + q]) * lz : lz;
            if (A.G2) {
                const long long jo = (long long)s * g.vol + o + q, js = (long long)g.n_shots * g.vol;
                if (mx) g2[q] -= lx * A.img_j[jo];
                if (my) g2[q] -= ly * A.img_j[js + jo];
                if (mz) g2[q] -= lz * A.img_j[2 * js + jo];
            }
        }
    }
    if (A.G2) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (x0 + q < g.Nx) neumaier3(A.G2[o + q], A.C2[o + q], g2[q]);
    }
}

__global__ void __launch_bounds__(128) adj_p3_kernel(const AdjArgs3 A)
{
    const Geo3 &g = A.g;
    const int x0 = 4 * (blockIdx.x * 32 + threadIdx.x);
    const int y = blockIdx.y * 4 + threadIdx.y;
    const int z = blockIdx.z;
    if (x0 >= g.Nx || y >= g.Ny) return;
    const long long o = (long long)z * g.plane + (long long)y * g.pitch + x0;
    float g1[4] = {0.f, 0.f, 0.f, 0.f};
    for (int s = 0; s < g.n_shots; ++s) {
        const float *L = A.lam_in + (long long)s * 4 * g.vol;     // lp' and lam_c'
        float *O = A.lam_out + (long long)s * 4 * g.vol;
        auto u = [&](int zz, int yy, int xx) {
            return in_p(g, zz, yy, xx) ? at3(g, A.a1, zz, yy, xx) * at3(g, L, zz, yy, xx) : 0.f;
        };
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int x = x0 + q;
            if (x >= g.Nx) break;
            const float lp = L[o + q];
            const bool mp = in_p(g, z, y, x);
            O[o + q] = mp ? (1.f - A.k1[o + q]) * lp : lp;
            if (mp) g1[q] += lp * A.img_i[(long long)s * g.vol + o + q];
            // lam_c = lam_c' - D_c^T u
            O[g.vol + o + q] = L[g.vol + o + q] -
                               (kC1 * (u(z, y, x) - u(z, y, x + 1)) + kC2 * (u(z, y, x - 1) - u(z, y, x + 2)));
            O[2 * g.vol + o + q] = L[2 * g.vol + o + q] -
                                   (kC1 * (u(z, y, x) - u(z, y + 1, x)) + kC2 * (u(z, y - 1, x) - u(z, y + 2, x)));
            O[3 * g.vol + o + q] = L[3 * g.vol + o + q] -
                                   (kC1 * (u(z, y, x) - u(z + 1, y, x)) + kC2 * (u(z - 1, y, x) - u(z + 2, y, x)));
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
        if (x0 + q < g.Nx) neumaier3(A.G1[o + q], A.C1[o + q], g1[q]);
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
