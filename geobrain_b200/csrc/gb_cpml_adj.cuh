// Adjoint (reverse time) of the CPML forward step, with the zero-lag imaging
// condition.  The CPML option is this library's extension; the forward it
// inverts is fwd_body's CPML branches:
//
//   psi_px' = bx psi_px + ax Dx(vx),  psi_pz' = bz psi_pz + az Dz(vz)      (p mask)
//   p'      = p - a1 ((Dx + psi_px') + (Dz + psi_pz'))  (+ source)
//   p'[fs-1] = -p'[fs+1]                                                 (free surface)
//   psi_vx' = bxh psi_vx + axh Gx(p'),  vx' = vx - a2 (Gx + psi_vx')      (vx mask)
//   psi_vz' = bzh psi_vz + azh Gz(p'),  vz' = vz - a2 (Gz + psi_vz')      (vz mask)
//   vz'[fs-1] = vz'[fs]
//
// With b = 1 + a these read p' = p - a1 (bx (Dx + psi_px) + bz (Dz + psi_pz))
// and vx' = vx - a2 bxh (Gx + psi_vx), which give the transposes below.  The
// adjoint state lam (unscaled) of the seven fields lives in ping-pong
// buffers [S][7][plane] (p, vx, vz, psi_px, psi_pz, psi_vx, psi_vz).  Per
// step, in reverse order of the forward:
//
//   inject   lam[receiver] += dL/dtrace[s, n, r]
//   fold     lam_vz[fs] += lam_vz[fs-1], lam_vz[fs-1] = 0
//   adj_v:   lam_p  += Gx^T(wx) + Gz^T(wz),  wx = M_vx (axh lam_psi_vx - a2 bxh lam_vx)
//            lam_psi_vx <- M_vx (bxh lam_psi_vx - a2 bxh lam_vx)   (likewise z)
//            G2 += a2 (lam_vx Jx + lam_vz Jz)
//   fold     lam_p[fs+1] -= lam_p[fs-1], lam_p[fs-1] = 0
//   adj_p:   lam_vx += Dx^T(ux),  ux = M_p (ax lam_psi_px - a1 bx lam_p)   (likewise z,
//            also on the vz mirror row, which the next step's fold takes)
//            lam_psi_px <- M_p (bx lam_psi_px - a1 bx lam_p)
//            G1 += a1 lam_p I
//
// with (Gx^T w)[i] = sum_k c_k (w[i-1-k] - w[i+k]) and
// (Dx^T u)[i] = sum_k c_k (u[i-k] - u[i+1+k]) along each axis.  I = -((Dx +
// psi_px') + (Dz + psi_pz')) and J = G + psi_v' are the imaging fields the
// forward stores.  As in the damping adjoint, cells outside the update
// masks never depend on the model, so their adjoint is dropped; the mirror
// rows are folded instead.  G1 and G2 hold a1 dL/da1 and -a2 dL/da2, which
// grad_finish_kernel turns into dL/dvp and dL/drho.  These are plain
// gather kernels (one cell per thread, all shots, neighbours through L1):
// the CPML gradient is an opt-in path, written for clarity.
#pragma once

#include "gb_adj.cuh"

namespace gb {

constexpr int kCpmlFields = 7;

struct CpmlAdjArgs {
    StepGeom g;
    const float *a1, *a2;
    const float *prof;          // [bz, az, bzh, azh][Nz] then [bx, ax, bxh, axh][pitch]
    const float *lin;           // [S][7][plane]
    float *lout;
    const float *img;           // this step's I [S][plane], then Jx, Jz at img_field_stride
    long long img_field_stride;
    int img_fmt;
    float *G1, *C1, *G2, *C2;   // one [plane] each (group 0 of the gradient planes)
    int free_surface;
};

__device__ __forceinline__ bool cp_in_p(const StepGeom &g, int z, int x)
{
    return z >= g.p_r0 && z <= g.p_r1 && x >= g.p_c0 && x <= g.p_c1;
}
__device__ __forceinline__ bool cp_in_vx(const StepGeom &g, int z, int x)
{
    return z >= g.vx_r0 && z <= g.vx_r1 && x >= g.vx_c0 && x <= g.vx_c1;
}
__device__ __forceinline__ bool cp_in_vz(const StepGeom &g, int z, int x)
{
    return z >= g.vz_r0 && z <= g.vz_r1 && x >= g.vz_c0 && x <= g.vz_c1;
}

// one imaging value at element offset o
__device__ __forceinline__ float cp_img(const float *base, long long o, int fmt)
{
    const float4 v = decode_img4(load_img_raw(base, o & ~3LL, fmt), fmt);
    return at(v, (int)(o & 3));
}

// adjoint receiver injection: lam[field][receiver cell] += res[s][it][r]
__global__ void cpml_inject_kernel(const StepGeom g, float *lam, const int2 *rcv, const float *res_p,
                                   const float *res_vx, const float *res_vz, int it)
{
    const long long n = (long long)g.n_shots * g.n_rcv;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / g.n_rcv), r = (int)(i % g.n_rcv);
        const long long o = (long long)rcv[r].x * g.pitch + rcv[r].y;
        float *L = lam + (long long)s * kCpmlFields * g.plane;
        const long long t = ((long long)s * g.nt + it) * g.n_rcv + r;
        if (res_p) atomicAdd(L + o, res_p[t]);   // receivers may share a cell
        if (res_vx) atomicAdd(L + g.plane + o, res_vx[t]);
        if (res_vz) atomicAdd(L + 2 * g.plane + o, res_vz[t]);
    }
}

// free-surface fold of field f: row fs-1 into row fs-1+to with sign, then cleared
__global__ void cpml_fold_kernel(const StepGeom g, float *lam, int field, int to, float sign)
{
    const long long n = (long long)g.n_shots * g.Nx;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / g.Nx), x = (int)(i % g.Nx);
        float *F = lam + ((long long)s * kCpmlFields + field) * g.plane;
        const long long m = (long long)(g.fs - 1) * g.pitch + x;
        F[m + (long long)to * g.pitch] += sign * F[m];
        F[m] = 0.f;
    }
}

// block (128, 2): one cell per thread, looping over the shots, so each cell
// of the gradient planes has one owner
template <int R>
__global__ void __launch_bounds__(256) cpml_adj_v_kernel(const CpmlAdjArgs A)
{
    const StepGeom &g = A.g;
    const int x = blockIdx.x * 128 + threadIdx.x;
    const int z = blockIdx.y * 2 + threadIdx.y;
    if (x >= g.Nx || z >= g.Nz) return;
    const long long o = (long long)z * g.pitch + x;
    const float *bzh = A.prof + 2 * g.Nz, *azh = A.prof + 3 * g.Nz;
    const float *bxh = A.prof + 4 * g.Nz + 2 * g.pitch, *axh = A.prof + 4 * g.Nz + 3 * g.pitch;
    // lam_p is kept on the p mask and on the mirror row (folded next)
    const bool mp = cp_in_p(g, z, x) || (A.free_surface && z == g.fs - 1);
    const bool mvx = cp_in_vx(g, z, x), mvz = cp_in_vz(g, z, x);
    const float a2 = A.a2[o];
    float g2 = 0.f, c2 = 0.f;
    for (int s = 0; s < g.n_shots; ++s) {
        const float *L = A.lin + (long long)s * kCpmlFields * g.plane;
        float *O = A.lout + (long long)s * kCpmlFields * g.plane;
        const float *Lvx = L + g.plane, *Lvz = L + 2 * g.plane, *Lsvx = L + 5 * g.plane, *Lsvz = L + 6 * g.plane;
        float lp = 0.f;
        if (mp) {
            float t = 0.f;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                float wm = 0.f, wp = 0.f, zm = 0.f, zp = 0.f;
                const int jm = x - 1 - k, jp = x + k, im = z - 1 - k, ip = z + k;
                if (cp_in_vx(g, z, jm)) {
                    const long long q = (long long)z * g.pitch + jm;
                    wm = axh[jm] * Lsvx[q] - A.a2[q] * bxh[jm] * Lvx[q];
                }
                if (cp_in_vx(g, z, jp)) {
                    const long long q = (long long)z * g.pitch + jp;
                    wp = axh[jp] * Lsvx[q] - A.a2[q] * bxh[jp] * Lvx[q];
                }
                if (cp_in_vz(g, im, x)) {
                    const long long q = (long long)im * g.pitch + x;
                    zm = azh[im] * Lsvz[q] - A.a2[q] * bzh[im] * Lvz[q];
                }
                if (cp_in_vz(g, ip, x)) {
                    const long long q = (long long)ip * g.pitch + x;
                    zp = azh[ip] * Lsvz[q] - A.a2[q] * bzh[ip] * Lvz[q];
                }
                t += g.c[k] * ((wm - wp) + (zm - zp));
            }
            lp = L[o] + t;
        }
        const float lvx = mvx ? Lvx[o] : 0.f, lvz = mvz ? Lvz[o] : 0.f;
        O[o] = lp;
        O[g.plane + o] = lvx;
        O[2 * g.plane + o] = lvz;
        O[3 * g.plane + o] = L[3 * g.plane + o];
        O[4 * g.plane + o] = L[4 * g.plane + o];
        O[5 * g.plane + o] = mvx ? bxh[x] * Lsvx[o] - a2 * bxh[x] * lvx : 0.f;
        O[6 * g.plane + o] = mvz ? bzh[z] * Lsvz[o] - a2 * bzh[z] * lvz : 0.f;
        if (A.G2 && (mvx || mvz)) {
            const long long io = (long long)s * g.plane + o;
            const float jx = mvx ? cp_img(A.img, A.img_field_stride + io, A.img_fmt) : 0.f;
            const float jz = mvz ? cp_img(A.img, 2 * A.img_field_stride + io, A.img_fmt) : 0.f;
            neumaier_add(g2, c2, a2 * (lvx * jx + lvz * jz));
        }
    }
    if (A.G2) neumaier_add(A.G2[o], A.C2[o], g2 + c2);
}

template <int R>
__global__ void __launch_bounds__(256) cpml_adj_p_kernel(const CpmlAdjArgs A)
{
    const StepGeom &g = A.g;
    const int x = blockIdx.x * 128 + threadIdx.x;
    const int z = blockIdx.y * 2 + threadIdx.y;
    if (x >= g.Nx || z >= g.Nz) return;
    const long long o = (long long)z * g.pitch + x;
    const float *bz = A.prof, *az = A.prof + g.Nz;
    const float *bx = A.prof + 4 * g.Nz, *ax = A.prof + 4 * g.Nz + g.pitch;
    // lam_vz is kept on the vz mask and on the mirror row: the p update read
    // vz[fs-1], which the previous step's mirror set (folded next step)
    const bool mp = cp_in_p(g, z, x), mvx = cp_in_vx(g, z, x);
    const bool mvz = cp_in_vz(g, z, x) || (A.free_surface && z == g.fs - 1);
    const float a1 = A.a1[o];
    float g1 = 0.f, c1 = 0.f;
    for (int s = 0; s < g.n_shots; ++s) {
        const float *L = A.lin + (long long)s * kCpmlFields * g.plane;
        float *O = A.lout + (long long)s * kCpmlFields * g.plane;
        const float *Lp = L, *Lspx = L + 3 * g.plane, *Lspz = L + 4 * g.plane;
        const float lp = mp ? Lp[o] : 0.f;
        float lvx = 0.f, lvz = 0.f;
        if (mvx) {
            // Dx^T: sum_k c_k (ux[x-k] - ux[x+1+k]),  ux[j] = M_p (ax lam_psi_px - a1 bx lam_p)
            float t = 0.f;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                float um = 0.f, up = 0.f;
                const int jm = x - k, jp = x + 1 + k;
                if (cp_in_p(g, z, jm)) {
                    const long long q = (long long)z * g.pitch + jm;
                    um = ax[jm] * Lspx[q] - A.a1[q] * bx[jm] * Lp[q];
                }
                if (cp_in_p(g, z, jp)) {
                    const long long q = (long long)z * g.pitch + jp;
                    up = ax[jp] * Lspx[q] - A.a1[q] * bx[jp] * Lp[q];
                }
                t += g.c[k] * (um - up);
            }
            lvx = L[g.plane + o] + t;
        }
        if (mvz) {
            float t = 0.f;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                float um = 0.f, up = 0.f;
                const int im = z - k, ip = z + 1 + k;
                if (cp_in_p(g, im, x)) {
                    const long long q = (long long)im * g.pitch + x;
                    um = az[im] * Lspz[q] - A.a1[q] * bz[im] * Lp[q];
                }
                if (cp_in_p(g, ip, x)) {
                    const long long q = (long long)ip * g.pitch + x;
                    up = az[ip] * Lspz[q] - A.a1[q] * bz[ip] * Lp[q];
                }
                t += g.c[k] * (um - up);
            }
            lvz = L[2 * g.plane + o] + t;
        }
        O[o] = lp;
        O[g.plane + o] = lvx;
        O[2 * g.plane + o] = lvz;
        O[3 * g.plane + o] = mp ? bx[x] * Lspx[o] - a1 * bx[x] * lp : 0.f;
        O[4 * g.plane + o] = mp ? bz[z] * Lspz[o] - a1 * bz[z] * lp : 0.f;
        O[5 * g.plane + o] = L[5 * g.plane + o];
        O[6 * g.plane + o] = L[6 * g.plane + o];
        if (mp) neumaier_add(g1, c1, a1 * lp * cp_img(A.img, (long long)s * g.plane + o, A.img_fmt));
    }
    neumaier_add(A.G1[o], A.C1[o], g1 + c1);
}

}  // namespace gb
