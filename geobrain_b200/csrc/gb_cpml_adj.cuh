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
// adjoint state lam (unscaled) of the seven fields lives in one buffer
// [S][11][plane]: lam_p, lam_vx, lam_vz updated in place, and two slots of
// each memory variable used in turn (the kernels read those at neighbours
// while they write them).  Per step, in reverse order of the forward:
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
// grad_finish_kernel turns into dL/dvp and dL/drho.  The kernels gather
// (4 adjacent cells per thread, all shots, neighbours through L1) with the
// masks folded into coefficient planes built once per gradient.
#pragma once

#include "gb_adj.cuh"

namespace gb {

constexpr int kCpmlPlanes = 11;   // the adjoint state planes of one shot (below)

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

// adjoint receiver injection: lam[field][receiver cell] += res[s][it][r]
__global__ void cpml_inject_kernel(const StepGeom g, float *lam, const int2 *rcv, const float *res_p,
                                   const float *res_vx, const float *res_vz, int it)
{
    const long long n = (long long)g.n_shots * g.n_rcv;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / g.n_rcv), r = (int)(i % g.n_rcv);
        const long long o = (long long)rcv[r].x * g.pitch + rcv[r].y;
        float *L = lam + (long long)s * kCpmlPlanes * g.plane;
        const long long t = ((long long)s * g.nt + it) * g.n_rcv + r;
        if (res_p) atomicAdd(L + o, res_p[t]);   // receivers may share a cell
        if (res_vx) atomicAdd(L + g.plane + o, res_vx[t]);
        if (res_vz) atomicAdd(L + 2 * g.plane + o, res_vz[t]);
    }
}

// dL/dwavelet[s, it] = dt * lam_p at the source cell, read between adj_v and
// adj_p (lam_p is then the adjoint of p just after the source was added)
__global__ void cpml_wavelet_grad_kernel(const StepGeom g, const float *lam, const int *src_z, const int *src_x,
                                         float *grad_wavelet, int it)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.n_shots) return;
    const long long o = (long long)src_z[s] * g.pitch + src_x[s];
    grad_wavelet[(long long)s * g.nt + it] = g.dt * lam[(long long)s * kCpmlPlanes * g.plane + o];
}

// free-surface fold of field f: row fs-1 into row fs-1+to with sign, then cleared
__global__ void cpml_fold_kernel(const StepGeom g, float *lam, int field, int to, float sign)
{
    const long long n = (long long)g.n_shots * g.Nx;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / g.Nx), x = (int)(i % g.Nx);
        float *F = lam + ((long long)s * kCpmlPlanes + field) * g.plane;
        const long long m = (long long)(g.fs - 1) * g.pitch + x;
        F[m + (long long)to * g.pitch] += sign * F[m];
        F[m] = 0.f;
    }
}

// Coefficient planes of the two adjoint kernels, with the update masks
// folded in (zero off the mask), built once per gradient:
//   [0] WX = M_vx a2 bxh  [1] AX = M_vx axh  [2] BX = M_vx bxh
//   [3] WZ = M_vz a2 bzh  [4] AZ = M_vz azh  [5] BZ = M_vz bzh
//   [6] UX = M_p a1 bx    [7] PX = M_p ax    [8] QX = M_p bx
//   [9] UZ = M_p a1 bz    [10] PZ = M_p az   [11] QZ = M_p bz
constexpr int kCpmlCoefPlanes = 12;

__global__ void cpml_adj_coef_kernel(const StepGeom g, const float *a1, const float *a2, const float *prof,
                                     float *cp)
{
    const float *bz = prof, *az = prof + g.Nz, *bzh = prof + 2 * g.Nz, *azh = prof + 3 * g.Nz;
    const float *bx = prof + 4 * g.Nz, *ax = bx + g.pitch, *bxh = bx + 2 * g.pitch, *axh = bx + 3 * g.pitch;
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < g.plane; o += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(o / g.pitch), x = (int)(o % g.pitch);
        const bool mvx = x < g.Nx && cp_in_vx(g, z, x), mvz = x < g.Nx && cp_in_vz(g, z, x);
        const bool mp = x < g.Nx && cp_in_p(g, z, x);
        const float v[kCpmlCoefPlanes] = {
            mvx ? a2[o] * bxh[x] : 0.f, mvx ? axh[x] : 0.f, mvx ? bxh[x] : 0.f,
            mvz ? a2[o] * bzh[z] : 0.f, mvz ? azh[z] : 0.f, mvz ? bzh[z] : 0.f,
            mp ? a1[o] * bx[x] : 0.f,   mp ? ax[x] : 0.f,   mp ? bx[x] : 0.f,
            mp ? a1[o] * bz[z] : 0.f,   mp ? az[z] : 0.f,   mp ? bz[z] : 0.f};
#pragma unroll
        for (int i = 0; i < kCpmlCoefPlanes; ++i) cp[i * g.plane + o] = v[i];
    }
}

// The adjoint state of one shot: [kCpmlPlanes][plane].  lam_p, lam_vx and
// lam_vz have one slot each and are updated in place (neither kernel reads
// at its neighbours a field it writes); the memory variables, which the
// kernels read at neighbours and rewrite, have two slots each, used in turn:
constexpr int kLamP = 0, kLamVX = 1, kLamVZ = 2;
constexpr int kPsiP0 = 3;   // psi_px, psi_pz, slot 0 at 3, 4 and slot 1 at 5, 6
constexpr int kPsiV0 = 7;   // psi_vx, psi_vz, slot 0 at 7, 8 and slot 1 at 9, 10

// Ask L2 for the next shot's fields of this thread's cells while the current
// shot computes (the loads of one shot alone leave DRAM idle between shots
// at 12-16 resident warps per SM).
__device__ __forceinline__ void cp_prefetch(const float *L, long long P, long long o, int f0, int f1)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(L + o));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(L + P + o));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(L + 2 * P + o));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(L + f0 * P + o));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(L + f1 * P + o));
}

struct CpmlAdjArgs4 {
    StepGeom g;
    const float *a1, *a2;
    const float *cp;            // the kCpmlCoefPlanes planes
    float *lam;                 // [S][kCpmlPlanes][plane]
    int psi_in, psi_out;        // first plane of the memory-variable slot read / written
    const float *img;           // this step's I [S][plane], then Jx, Jz at img_field_stride
    long long img_field_stride;
    int img_fmt;
    float *G1, *C1, *G2, *C2;   // [n_groups][plane] each: shot group g adds into plane g
    int free_surface;
};

__device__ __forceinline__ float4 cp_ld4(const float *base, long long o, bool ok)
{
    return ok ? __ldg(reinterpret_cast<const float4 *>(base + o)) : zero4();
}
// plain load, for the fields a kernel also writes (in place, own cells only)
__device__ __forceinline__ float4 cp_ldw4(const float *base, long long o)
{
    return *reinterpret_cast<const float4 *>(base + o);
}
__device__ __forceinline__ float4 fms4(const float4 &a, const float4 &x, const float4 &b, const float4 &y)
{
    // a x - b y per lane
    return make_float4(a.x * x.x - b.x * y.x, a.y * x.y - b.y * y.y, a.z * x.z - b.z * y.z, a.w * x.w - b.w * y.w);
}

// Rows per thread of the two adjoint kernels: a thread updates 4 adjacent
// cells of kCpLZ consecutive rows and keeps the z-direction operand of its
// rows and their 2R - 1 neighbours in a register window, so a row of the
// memory variable and its field is read once per kCpLZ output rows (2R
// times per row with one row per thread).  Two rows: at four the window and
// the per-row gradient sums spilled (280-476 bytes at 8th order).
constexpr int kCpLZ = 2;

// block (32, 4), grid (x, z, shot group): a thread owns 4 x kCpLZ cells and
// loops over the shots of its group, so each cell of the group's gradient
// planes has one owner.  Reads lam_vx, lam_vz and the psi_v slot psi_in (at
// neighbours), writes lam_p in place and the psi_v slot psi_out.
template <int R>
__global__ void __launch_bounds__(128, 4) cpml_adj_v_kernel(const CpmlAdjArgs4 A)
{
    constexpr int LZ = kCpLZ, NWZ = LZ + 2 * R - 1;
    const StepGeom &g = A.g;
    const int x0 = 4 * (blockIdx.x * 32 + threadIdx.x);
    const int z0 = (blockIdx.y * 4 + threadIdx.y) * LZ;
    if (x0 >= g.Nx || z0 >= g.Nz) return;
    const int grp = blockIdx.z, s0 = grp * g.shots_per_cta, s1 = min(g.n_shots, s0 + g.shots_per_cta);
    const long long P = g.plane;
    const float *WX = A.cp, *AX = A.cp + P, *BX = A.cp + 2 * P, *WZ = A.cp + 3 * P, *AZ = A.cp + 4 * P,
                *BZ = A.cp + 5 * P;
    const bool lok = x0 >= 4, rok = x0 + 4 < g.pitch;
    float g2[LZ][4], c2[LZ][4];
#pragma unroll
    for (int u = 0; u < LZ; ++u)
#pragma unroll
        for (int q = 0; q < 4; ++q) g2[u][q] = c2[u][q] = 0.f;
    for (int s = s0; s < s1; ++s) {
        float *L = A.lam + (long long)s * kCpmlPlanes * P;
        const float *Lvx = L + kLamVX * P, *Lvz = L + kLamVZ * P;
        const float *Lsvx = L + A.psi_in * P, *Lsvz = L + (A.psi_in + 1) * P;
        if (s + 1 < s1)
#pragma unroll
            for (int u = 0; u < LZ; ++u)
                if (z0 + u < g.Nz)
                    cp_prefetch(L + kCpmlPlanes * P, P, (long long)(z0 + u) * g.pitch + x0, A.psi_in, A.psi_in + 1);
        // wz = AZ lam_psi_vz - WZ lam_vz on rows z0-R .. z0+LZ+R-2
        float4 wz[NWZ];
#pragma unroll
        for (int t = 0; t < NWZ; ++t) {
            const int zr = z0 - R + t;
            const long long q = (long long)zr * g.pitch + x0;
            wz[t] = (zr >= 0 && zr < g.Nz)
                        ? fms4(cp_ld4(AZ, q, true), cp_ld4(Lsvz, q, true), cp_ld4(WZ, q, true), cp_ld4(Lvz, q, true))
                        : zero4();
        }
#pragma unroll
        for (int u = 0; u < LZ; ++u) {
            const int z = z0 + u;
            if (z >= g.Nz) break;
            const long long o = (long long)z * g.pitch + x0;
            // wx = AX lam_psi_vx - WX lam_vx at x0-4 .. x0+7
            float wx[12];
            {
                const float4 l = fms4(cp_ld4(AX, o - 4, lok), cp_ld4(Lsvx, o - 4, lok), cp_ld4(WX, o - 4, lok),
                                      cp_ld4(Lvx, o - 4, lok));
                const float4 c = fms4(cp_ld4(AX, o, true), cp_ld4(Lsvx, o, true), cp_ld4(WX, o, true),
                                      cp_ld4(Lvx, o, true));
                const float4 r = fms4(cp_ld4(AX, o + 4, rok), cp_ld4(Lsvx, o + 4, rok), cp_ld4(WX, o + 4, rok),
                                      cp_ld4(Lvx, o + 4, rok));
                const float t[12] = {l.x, l.y, l.z, l.w, c.x, c.y, c.z, c.w, r.x, r.y, r.z, r.w};
#pragma unroll
                for (int i = 0; i < 12; ++i) wx[i] = t[i];
            }
            const float4 lp = cp_ldw4(L, o), lvx = cp_ld4(Lvx, o, true), lvz = cp_ld4(Lvz, o, true);
            const float4 lsvx = cp_ld4(Lsvx, o, true), lsvz = cp_ld4(Lsvz, o, true);
            float4 op, mvxv, mvzv;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int x = x0 + q;
                const bool mp = x < g.Nx && (cp_in_p(g, z, x) || (A.free_surface && z == g.fs - 1));   // mirror row: folded next
                float t = 0.f;
#pragma unroll
                for (int k = 0; k < R; ++k)
                    t += g.c[k] *
                         ((wx[q + 3 - k] - wx[q + 4 + k]) + (at(wz[u + R - 1 - k], q) - at(wz[u + R + k], q)));
                at(op, q) = mp ? at(lp, q) + t : 0.f;
                at(mvxv, q) = (x < g.Nx && cp_in_vx(g, z, x)) ? at(lvx, q) : 0.f;
                at(mvzv, q) = (x < g.Nx && cp_in_vz(g, z, x)) ? at(lvz, q) : 0.f;
            }
            stg4(L + o, op);
            stg4(L + A.psi_out * P + o, fms4(cp_ld4(BX, o, true), lsvx, cp_ld4(WX, o, true), lvx));
            stg4(L + (A.psi_out + 1) * P + o, fms4(cp_ld4(BZ, o, true), lsvz, cp_ld4(WZ, o, true), lvz));
            if (A.G2) {
                const float4 a2 = cp_ld4(A.a2, o, true);
                const long long io = (long long)s * P + o;
                const float4 jx = decode_img4(load_img_raw(A.img, A.img_field_stride + io, A.img_fmt), A.img_fmt);
                const float4 jz =
                    decode_img4(load_img_raw(A.img, 2 * A.img_field_stride + io, A.img_fmt), A.img_fmt);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    neumaier_add(g2[u][q], c2[u][q], at(a2, q) * (at(mvxv, q) * at(jx, q) + at(mvzv, q) * at(jz, q)));
            }
        }
    }
    if (A.G2) {
#pragma unroll
        for (int u = 0; u < LZ; ++u) {
            const long long o = (long long)(z0 + u) * g.pitch + x0 + (long long)grp * P;
            if (z0 + u < g.Nz)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (x0 + q < g.Nx) neumaier_add(A.G2[o + q], A.C2[o + q], g2[u][q] + c2[u][q]);
        }
    }
}

// Reads lam_p and the psi_p slot psi_in (at neighbours), writes lam_vx and
// lam_vz in place and the psi_p slot psi_out (the layout of
// cpml_adj_v_kernel: 4 x kCpLZ cells per thread, shot groups in grid z).
template <int R>
__global__ void __launch_bounds__(128, 4) cpml_adj_p_kernel(const CpmlAdjArgs4 A)
{
    constexpr int LZ = kCpLZ, NWZ = LZ + 2 * R - 1;
    const StepGeom &g = A.g;
    const int x0 = 4 * (blockIdx.x * 32 + threadIdx.x);
    const int z0 = (blockIdx.y * 4 + threadIdx.y) * LZ;
    if (x0 >= g.Nx || z0 >= g.Nz) return;
    const int grp = blockIdx.z, s0 = grp * g.shots_per_cta, s1 = min(g.n_shots, s0 + g.shots_per_cta);
    const long long P = g.plane;
    const float *UX = A.cp + 6 * P, *PX = A.cp + 7 * P, *QX = A.cp + 8 * P, *UZ = A.cp + 9 * P,
                *PZ = A.cp + 10 * P, *QZ = A.cp + 11 * P;
    const bool lok = x0 >= 4, rok = x0 + 4 < g.pitch;
    float g1[LZ][4], c1[LZ][4];
#pragma unroll
    for (int u = 0; u < LZ; ++u)
#pragma unroll
        for (int q = 0; q < 4; ++q) g1[u][q] = c1[u][q] = 0.f;
    for (int s = s0; s < s1; ++s) {
        float *L = A.lam + (long long)s * kCpmlPlanes * P;
        const float *Lspx = L + A.psi_in * P, *Lspz = L + (A.psi_in + 1) * P;
        if (s + 1 < s1)
#pragma unroll
            for (int u = 0; u < LZ; ++u)
                if (z0 + u < g.Nz)
                    cp_prefetch(L + kCpmlPlanes * P, P, (long long)(z0 + u) * g.pitch + x0, A.psi_in, A.psi_in + 1);
        // uz = PZ lam_psi_pz - UZ lam_p on rows z0-R+1 .. z0+LZ+R-1
        float4 uz[NWZ];
#pragma unroll
        for (int t = 0; t < NWZ; ++t) {
            const int zr = z0 - R + 1 + t;
            const long long q = (long long)zr * g.pitch + x0;
            uz[t] = (zr >= 0 && zr < g.Nz)
                        ? fms4(cp_ld4(PZ, q, true), cp_ld4(Lspz, q, true), cp_ld4(UZ, q, true), cp_ld4(L, q, true))
                        : zero4();
        }
#pragma unroll
        for (int u = 0; u < LZ; ++u) {
            const int z = z0 + u;
            if (z >= g.Nz) break;
            const long long o = (long long)z * g.pitch + x0;
            // ux = PX lam_psi_px - UX lam_p at x0-4 .. x0+7
            float ux[12];
            {
                const float4 l = fms4(cp_ld4(PX, o - 4, lok), cp_ld4(Lspx, o - 4, lok), cp_ld4(UX, o - 4, lok),
                                      cp_ld4(L, o - 4, lok));
                const float4 c = fms4(cp_ld4(PX, o, true), cp_ld4(Lspx, o, true), cp_ld4(UX, o, true),
                                      cp_ld4(L, o, true));
                const float4 r = fms4(cp_ld4(PX, o + 4, rok), cp_ld4(Lspx, o + 4, rok), cp_ld4(UX, o + 4, rok),
                                      cp_ld4(L, o + 4, rok));
                const float t[12] = {l.x, l.y, l.z, l.w, c.x, c.y, c.z, c.w, r.x, r.y, r.z, r.w};
#pragma unroll
                for (int i = 0; i < 12; ++i) ux[i] = t[i];
            }
            const float4 lp = cp_ld4(L, o, true), lvx = cp_ldw4(L + kLamVX * P, o), lvz = cp_ldw4(L + kLamVZ * P, o);
            const float4 lspx = cp_ld4(Lspx, o, true), lspz = cp_ld4(Lspz, o, true);
            float4 ovx, ovz;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int x = x0 + q;
                float tx = 0.f, tz = 0.f;
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    tx += g.c[k] * (ux[q + 4 - k] - ux[q + 5 + k]);
                    tz += g.c[k] * (at(uz[u + R - 1 - k], q) - at(uz[u + R + k], q));
                }
                // the p update read vz[fs-1], which the previous step's mirror set (folded next step)
                const bool mvz = x < g.Nx && (cp_in_vz(g, z, x) || (A.free_surface && z == g.fs - 1));
                at(ovx, q) = (x < g.Nx && cp_in_vx(g, z, x)) ? at(lvx, q) + tx : 0.f;
                at(ovz, q) = mvz ? at(lvz, q) + tz : 0.f;
            }
            stg4(L + kLamVX * P + o, ovx);
            stg4(L + kLamVZ * P + o, ovz);
            stg4(L + A.psi_out * P + o, fms4(cp_ld4(QX, o, true), lspx, cp_ld4(UX, o, true), lp));
            stg4(L + (A.psi_out + 1) * P + o, fms4(cp_ld4(QZ, o, true), lspz, cp_ld4(UZ, o, true), lp));
            const float4 a1 = cp_ld4(A.a1, o, true);
            const float4 im = decode_img4(load_img_raw(A.img, (long long)s * P + o, A.img_fmt), A.img_fmt);
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (x0 + q < g.Nx && cp_in_p(g, z, x0 + q))
                    neumaier_add(g1[u][q], c1[u][q], at(a1, q) * at(lp, q) * at(im, q));
        }
    }
#pragma unroll
    for (int u = 0; u < LZ; ++u) {
        const long long o = (long long)(z0 + u) * g.pitch + x0 + (long long)grp * P;
        if (z0 + u < g.Nz)
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (x0 + q < g.Nx) neumaier_add(A.G1[o + q], A.C1[o + q], g1[u][q] + c1[u][q]);
    }
}

}  // namespace gb
