// Fused adjoint time step (reverse time) with the zero-lag imaging condition.
//
// This is the exact discrete adjoint of fwd_step_kernel, i.e. of the
// reference step (geobrain/physics/wave/kernels/acoustic_2d.py:211-274), in
// scaled variables mu_p = alpha1 * lambda_p and mu_v = alpha2 * lambda_v,
// where lambda is the reverse-mode adjoint of the stored state.  In those
// variables the adjoint step has the same two-stencil shape as the forward:
//
//   inject  mu[receiver] += scale * dL/dtrace[s, n, r]          (adjoint of :272-274)
//   stage A (whole p rectangle):
//     mu_p  <- M_p ? mu_p + a1 * div(mu_vx, mu_vz) : 0           (adjoint of :244-265)
//              (free surface: row fs+1 also takes the mirror row's share)
//   stage B (tile):
//     mu_vx <- M_vx ? (1 - k2) mu_vx + a2 * dx(mu_p) : 0         (adjoint of :211-226)
//     mu_vz <- M_vz ? (1 - k3) mu_vz + a2 * dz(mu_p) : 0
//              (free surface: row fs also takes the virtual vz[fs-1] read)
//     mu_p  <- M_p ? (1 - k1) mu_p : 0
//     G1    += mu_p * I_n        I_n = -div(v^n), stored by the recompute
//     G2    += mu_vx * Jx_n + mu_vz * Jz_n   (only for the density gradient)
//
// Cells outside the update masks never depend on the model, so their adjoint
// is dropped (held at zero); that keeps every stencil read mask-free.
// dL/dvp and dL/drho follow from G1, G2 in grad_finish_kernel.
#pragma once

#include "gb_device.cuh"
#include "gb_fwd.cuh"

namespace gb {

struct AdjArgs {
    StepGeom g;
    int it;                                  // forward step whose adjoint this is
    const float *a1, *k1, *a2, *k2, *k3;
    float *out;                              // previous adjoint state [S][3][plane]
    const int *rcv_ptr;                      // CSR over tiles, receivers within the loaded rectangles
    const int4 *rcv_ent;                     // (padded z, padded x, receiver, 0)
    const float *res_p, *res_vx, *res_vz;    // [S][nt][n_rcv] or null
    const float *img;                        // [S][plane] I_n (and Jx, Jz planes after it when RHO)
    long long img_field_stride;              // distance between the I, Jx, Jz blocks
    float *G1, *C1, *G2, *C2;                // [n_groups][plane] sums and compensations
    int *err;
};

__device__ __forceinline__ void neumaier_add(float &s, float &c, float x)
{
    const float t = s + x;
    if (fabsf(s) >= fabsf(x))
        c += (s - t) + x;
    else
        c += (x - t) + s;
    s = t;
}

template <int R, int TZ, bool FS, bool RHO>
__global__ void __launch_bounds__(NTHR, 1)
adj_step_kernel(const __grid_constant__ CUtensorMap mP, const __grid_constant__ CUtensorMap mVX,
                const __grid_constant__ CUtensorMap mVZ, const AdjArgs A)
{
    using G = Geo<R, TZ>;
    const StepGeom &g = A.g;
    extern __shared__ __align__(128) float smem[];
    float *stage[2] = {smem, smem + G::STAGE_FL};
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * G::STAGE_FL);

    const int group = blockIdx.x % g.n_groups;
    const int tile = blockIdx.x / g.n_groups;
    const int z0 = (tile / g.tiles_x) * TZ;
    const int x0 = (tile % g.tiles_x) * TX;
    const int s0 = group * g.shots_per_cta;
    const int ns = min(g.n_shots - s0, g.shots_per_cta);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < 2 && k < ns; ++k)
            stage_loads<R>(&mP, &mVX, &mVZ, stage[k], &bars[k], G::STAGE_BYTES, x0, z0, s0 + k, G::P_FL,
                           G::VX_FL);
    }
    const int gx0 = x0 - 4 + 4 * lane;

    // per-thread partial sums over this CTA's shots (v-stage cells)
    float4 acc1[G::LV], acc2[G::LV];
#pragma unroll
    for (int u = 0; u < G::LV; ++u) {
        acc1[u] = zero4();
        acc2[u] = zero4();
    }

    for (int k = 0; k < ns; ++k) {
        const int s = s0 + k;
        const int b = k & 1;
        if (!__syncthreads_and(mbar_wait_bounded(&bars[b], (k >> 1) & 1))) {
            if (threadIdx.x == 0) {
                atomicExch(A.err, -4);
                if (k + 1 < ns) mbar_wait_bounded(&bars[b ^ 1], ((k + 1) >> 1) & 1);
            }
            return;
        }
        float *sP = stage[b];
        float *sVX = sP + G::P_FL;
        float *sVZ = sVX + G::VX_FL;

        // ---------------- adjoint sources at the receivers ------------------
        if (A.res_p || A.res_vx || A.res_vz) {
            const int e0 = A.rcv_ptr[tile], e1 = A.rcv_ptr[tile + 1];
            for (int e = e0 + threadIdx.x; e < e1; e += NTHR) {
                const int4 en = A.rcv_ent[e];
                const int gz = en.x, gx = en.y;
                const long long t = ((long long)s * g.nt + A.it) * g.n_rcv + en.z;
                const long long o = (long long)gz * g.pitch + gx;
                if (A.res_p && gz >= g.p_r0 && gz <= g.p_r1 && gx >= g.p_c0 && gx <= g.p_c1) {
                    const int r = gz - (z0 - R), c = gx - (x0 - 4);
                    if (r >= 0 && r < G::PR && c >= 0 && c < RW) atomicAdd(&sP[r * RW + c], A.a1[o] * A.res_p[t]);
                }
                if (A.res_vx && gz >= g.vx_r0 && gz <= g.vx_r1 && gx >= g.vx_c0 && gx <= g.vx_c1) {
                    const int r = gz - (z0 - R), c = gx - (x0 - 8);
                    if (r >= 0 && r < G::PR && c >= 0 && c < VXW)
                        atomicAdd(&sVX[r * VXW + c], A.a2[o] * A.res_vx[t]);
                }
                if (A.res_vz && gz >= g.vz_r0 && gz <= g.vz_r1 && gx >= g.vz_c0 && gx <= g.vz_c1) {
                    const int r = gz - (z0 - 2 * R), c = gx - (x0 - 4);
                    if (r >= 0 && r < G::ZR && c >= 0 && c < RW)
                        atomicAdd(&sVZ[r * RW + c], A.a2[o] * A.res_vz[t]);
                }
            }
            __syncthreads();
        }

        // ---------------- stage A: mu_p on the whole sP rectangle ----------
        {
            const int rb = warp * G::LP;
            const int rc = min(G::LP, G::PR - rb);
            float4 wz[G::LP + 2 * R - 1];
#pragma unroll
            for (int t = 0; t < G::LP + 2 * R - 1; ++t)
                wz[t] = (t < rc + 2 * R - 1) ? lds4(sVZ + (rb + t) * RW + 4 * lane) : zero4();
#pragma unroll
            for (int u = 0; u < G::LP; ++u) {
                if (u < rc) {
                    const int r = rb + u;
                    const int gz = z0 - R + r;
                    float4 pv = lds4(sP + r * RW + 4 * lane);
                    const bool row_in = gz >= g.p_r0 && gz <= g.p_r1;
                    if (row_in && (gx0 + 3 >= g.p_c0) && (gx0 <= g.p_c1)) {
                        float e[12];
                        {
                            const float4 e0 = lds4(sVX + r * VXW + 4 * lane);
                            const float4 e1 = lds4(sVX + r * VXW + 4 * lane + 4);
                            const float4 e2 = lds4(sVX + r * VXW + 4 * lane + 8);
                            e[0] = e0.x; e[1] = e0.y; e[2] = e0.z; e[3] = e0.w;
                            e[4] = e1.x; e[5] = e1.y; e[6] = e1.z; e[7] = e1.w;
                            e[8] = e2.x; e[9] = e2.y; e[10] = e2.z; e[11] = e2.w;
                        }
                        const float4 a1 = ldg4(A.a1 + (long long)gz * g.pitch + gx0);
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            float D = 0.f;
#pragma unroll
                            for (int kk = 0; kk < R; ++kk)
                                D += g.c[kk] * (((e[q + 4 + kk] - e[q + 3 - kk]) + at(wz[u + R + kk], q)) -
                                                at(wz[u + R - 1 - kk], q));
                            if (FS && gz == g.fs + 1) {
                                // share of the mirror row p[fs-1] = -p[fs+1]
                                float M = 0.f;
#pragma unroll
                                for (int kk = 0; kk < R; ++kk) M += g.c[kk] * at(wz[u + R - 2 + kk], q);
                                D -= M;
                            }
                            const int gx = gx0 + q;
                            at(pv, q) = (gx >= g.p_c0 && gx <= g.p_c1) ? at(pv, q) + at(a1, q) * D : 0.f;
                        }
                    } else {
                        pv = zero4();
                    }
                    sts4(sP + r * RW + 4 * lane, pv);
                }
            }
        }
        __syncthreads();

        // ---------------- stage B: tile --------------------------------------
        if (lane >= 1 && lane <= 30) {
            const int vb = warp * G::LV;
            const int vc = min(G::LV, TZ - vb);
            float4 wp[G::LV + 2 * R - 1];
#pragma unroll
            for (int t = 0; t < G::LV + 2 * R - 1; ++t)
                wp[t] = (t < vc + 2 * R - 1) ? lds4(sP + (vb + 1 + t) * RW + 4 * lane) : zero4();
#pragma unroll
            for (int u = 0; u < G::LV; ++u) {
                if (u < vc) {
                    const int rv = vb + u;
                    const int rr = rv + R;
                    const int gz = z0 + rv;
                    if (gz < g.Nz && gx0 < g.Nx) {
                        float f[12];
                        {
                            const float4 f0 = lds4(sP + rr * RW + 4 * lane - 4);
                            const float4 f1 = lds4(sP + rr * RW + 4 * lane);
                            const float4 f2 = lds4(sP + rr * RW + 4 * lane + 4);
                            f[0] = f0.x; f[1] = f0.y; f[2] = f0.z; f[3] = f0.w;
                            f[4] = f1.x; f[5] = f1.y; f[6] = f1.z; f[7] = f1.w;
                            f[8] = f2.x; f[9] = f2.y; f[10] = f2.z; f[11] = f2.w;
                        }
                        const float4 vx1 = lds4(sVX + rr * VXW + 4 * lane + 4);
                        const float4 vz1 = lds4(sVZ + (rv + 2 * R) * RW + 4 * lane);
                        const float4 mp1 = make_float4(f[4], f[5], f[6], f[7]);
                        float4 vx = zero4(), vz = zero4(), pp = zero4();
                        const long long o = (long long)gz * g.pitch + gx0;
                        const bool vx_row = gz >= g.vx_r0 && gz <= g.vx_r1;
                        const bool vz_row = gz >= g.vz_r0 && gz <= g.vz_r1;
                        const bool p_row = gz >= g.p_r0 && gz <= g.p_r1;
                        const bool any_v = (vx_row && gx0 + 3 >= g.vx_c0 && gx0 <= g.vx_c1) ||
                                           (vz_row && gx0 + 3 >= g.vz_c0 && gx0 <= g.vz_c1);
                        const bool any_p = p_row && gx0 + 3 >= g.p_c0 && gx0 <= g.p_c1;
                        if (any_v) {
                            const float4 a2 = ldg4(A.a2 + o);
                            const float4 k2 = ldg4(A.k2 + o);
                            const float4 k3 = ldg4(A.k3 + o);
                            float4 jx, jz;
                            if (RHO) {
                                jx = ldg4(A.img + (long long)s * g.plane + A.img_field_stride + o);
                                jz = ldg4(A.img + (long long)s * g.plane + 2 * A.img_field_stride + o);
                            }
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const int gx = gx0 + q;
                                if (vx_row && gx >= g.vx_c0 && gx <= g.vx_c1) {
                                    float D = 0.f;
#pragma unroll
                                    for (int kk = 0; kk < R; ++kk)
                                        D += g.c[kk] * (f[q + 5 + kk] - f[q + 4 - kk]);
                                    at(vx, q) = (1.f - at(k2, q)) * at(vx1, q) + at(a2, q) * D;
                                    if (RHO) at(acc2[u], q) += at(vx1, q) * at(jx, q);
                                }
                                if (vz_row && gx >= g.vz_c0 && gx <= g.vz_c1) {
                                    float D = 0.f;
#pragma unroll
                                    for (int kk = 0; kk < R; ++kk)
                                        D += g.c[kk] * (at(wp[u + R + kk], q) - at(wp[u + R - 1 - kk], q));
                                    if (FS && gz == g.fs) {
                                        // the p update reads vz[fs-1] as vz[fs]
#pragma unroll
                                        for (int kk = 0; kk < R; ++kk) D += g.c[kk] * at(wp[u + R - 1 + kk], q);
                                    }
                                    at(vz, q) = (1.f - at(k3, q)) * at(vz1, q) + at(a2, q) * D;
                                    if (RHO) at(acc2[u], q) += at(vz1, q) * at(jz, q);
                                }
                            }
                        }
                        if (any_p) {
                            const float4 k1 = ldg4(A.k1 + o);
                            const float4 im = ldg4(A.img + (long long)s * g.plane + o);
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const int gx = gx0 + q;
                                if (gx >= g.p_c0 && gx <= g.p_c1) {
                                    at(pp, q) = (1.f - at(k1, q)) * at(mp1, q);
                                    at(acc1[u], q) += at(mp1, q) * at(im, q);
                                }
                            }
                        }
                        float *outs = A.out + (long long)s * 3 * g.plane + o;
                        stg4(outs, pp);
                        stg4(outs + g.plane, vx);
                        stg4(outs + 2 * g.plane, vz);
                    }
                }
            }
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0 && k + 2 < ns) {
            stage_loads<R>(&mP, &mVX, &mVZ, stage[b], &bars[b], G::STAGE_BYTES, x0, z0, s + 2, G::P_FL,
                           G::VX_FL);
        }
    }

    // compensated accumulation of this step's partial sums into the group's
    // running totals (this CTA is their only writer for this tile)
    if (lane >= 1 && lane <= 30) {
        const int vb = warp * G::LV;
        const int vc = min(G::LV, TZ - vb);
#pragma unroll
        for (int u = 0; u < G::LV; ++u) {
            const int gz = z0 + vb + u;
            if (u < vc && gz >= g.p_r0 && gz <= g.p_r1 && gx0 < g.Nx) {
                const long long o = (long long)group * g.plane + (long long)gz * g.pitch + gx0;
                float4 s1 = *reinterpret_cast<float4 *>(A.G1 + o), c1 = *reinterpret_cast<float4 *>(A.C1 + o);
#pragma unroll
                for (int q = 0; q < 4; ++q) neumaier_add(at(s1, q), at(c1, q), at(acc1[u], q));
                stg4(A.G1 + o, s1);
                stg4(A.C1 + o, c1);
            }
            if (RHO && u < vc && gz < g.Nz && gx0 < g.Nx) {
                const long long o = (long long)group * g.plane + (long long)gz * g.pitch + gx0;
                float4 s2 = *reinterpret_cast<float4 *>(A.G2 + o), c2 = *reinterpret_cast<float4 *>(A.C2 + o);
#pragma unroll
                for (int q = 0; q < 4; ++q) neumaier_add(at(s2, q), at(c2, q), at(acc2[u], q));
                stg4(A.G2 + o, s2);
                stg4(A.C2 + o, c2);
            }
        }
    }
}

template <int R, int TZ>
constexpr size_t adj_smem_bytes()
{
    return 2 * Geo<R, TZ>::STAGE_BYTES + 16;
}

// dL/dvp and dL/drho on the (nz, nx) model: per padded cell
//   G1 = sum(mu_p1 * I), G2 = sum(mu_v1 * J) over groups (compensated),
//   dL/dc = 2 G1 / c, dL/dden = (G1 + G2) / den,
// then the adjoint of pad_model: each model cell collects every padded cell
// it was replicated into (acoustic_2d.py:55-64).
__global__ void grad_finish_kernel(const float *__restrict__ vp, const float *__restrict__ rho,
                                   const float *__restrict__ G1, const float *__restrict__ C1,
                                   const float *__restrict__ G2, const float *__restrict__ C2, int n_groups,
                                   long long plane, int nz, int nx, int pml, int pitch, float *grad_vp,
                                   float *grad_rho)
{
    const long long n = (long long)nz * nx;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int iz = (int)(idx / nx), ix = (int)(idx % nx);
        const float c = vp[idx], den = rho[idx];
        // padded rows / columns replicated from this cell
        const int r0 = iz == 0 ? 0 : iz + pml, r1 = iz == nz - 1 ? nz + 2 * pml - 1 : iz + pml;
        const int q0 = ix == 0 ? 0 : ix + pml, q1 = ix == nx - 1 ? nx + 2 * pml - 1 : ix + pml;
        float s1 = 0.f, e1 = 0.f, s2 = 0.f, e2 = 0.f;
        for (int i = r0; i <= r1; ++i)
            for (int j = q0; j <= q1; ++j) {
                const long long o = (long long)i * pitch + j;
                for (int gi = 0; gi < n_groups; ++gi) {
                    const long long og = gi * plane + o;
                    neumaier_add(s1, e1, G1[og]);
                    neumaier_add(s1, e1, C1[og]);
                    if (G2) {
                        neumaier_add(s2, e2, G2[og]);
                        neumaier_add(s2, e2, C2[og]);
                    }
                }
            }
        const float g1 = s1 + e1, g2 = s2 + e2;
        grad_vp[idx] = 2.f * g1 / c;
        if (grad_rho) grad_rho[idx] = (g1 + g2) / den;
    }
}

}  // namespace gb
