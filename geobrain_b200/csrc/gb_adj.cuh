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

#include "gb_fwd.cuh"

namespace gb {

struct AdjArgs {
    StepGeom g;
    int it;                                  // forward step whose adjoint this is
    const float *a1, *k1, *a2, *k2, *k3;
    const int *tile_fast;
    float *out;                              // previous adjoint state [S][3][plane]
    const int *rcv_ptr;                      // CSR over tiles, receivers within the loaded rectangles
    const int4 *rcv_ent;                     // (padded z, padded x, receiver, 0)
    const float *res_p, *res_vx, *res_vz;    // [S][nt][n_rcv] or null
    const float *img;                        // [S][plane] I_n (and Jx, Jz planes after it when RHO)
    long long img_field_stride;              // distance between the I, Jx, Jz blocks (elements)
    int img_fmt;                             // storage format of the imaging fields (kImg*)
    float *G1, *C1, *G2, *C2;                // [n_groups][plane] sums and compensations
    int grp0, grp_count;             // shot groups this launch covers
    const int *tile_order;           // the tiles in dispatch order (blockIdx / grp_count), or null: in index order
    int *err;
    // dL/dwavelet [S][nt] (or null): dt * lambda_p at the source cell after
    // stage A, i.e. the adjoint of p just after the source was added
    // (acoustic_2d.py:228-237); sources lie on the p mask (checked on the host)
    float *grad_wavelet;
    const int *src_z, *src_x;                // padded source cells
    // graph replay: with step_base set, the step is *step_base - it, and the
    // imaging fields of step t are at img_base + (t - img_t0) * img_step elements
    const int *step_base;
    float *img_base;
    long long img_step;
    int img_t0;
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

// IMGF: storage format of the imaging fields (kImg*), or -1 to read it from
// A.img_fmt at run time (batched launches, where it varies per model).
template <int R, int TZ, bool FS, bool RHO, int IMGF>
__device__ __forceinline__ void adj_body(const CUtensorMap *mP, const CUtensorMap *mVX, const CUtensorMap *mVZ,
                                         const CUtensorMap *mA1, const CUtensorMap *mA2,
                                         const AdjArgs &__restrict__ A, const int group, const int tile)
{
    const int img_fmt = IMGF >= 0 ? IMGF : A.img_fmt;
    using G = Geo<R, TZ>;
    using SM = StepSmem<R, TZ>;
    const StepGeom &__restrict__ g = A.g;
    extern __shared__ __align__(128) float smem[];
    float *sA1 = smem + 2 * G::STAGE_FL;
    float *sA2 = sA1 + SM::A1_FL;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sA1 + SM::COEF_FL);

    const int z0 = (tile / g.tiles_x) * TZ;
    const int x0 = (tile % g.tiles_x) * TX;
    const int s0 = group * g.shots_per_cta;
    const int ns = min(g.n_shots - s0, g.shots_per_cta);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1);
        fence_mbar_init();
    }
    grid_dependency_wait();
    grid_launch_dependents();
    // a CUDA graph replays the same launches for every chunk of steps (in
    // reverse); the chunk's top step comes from device memory
    const int it = A.step_base ? *reinterpret_cast<const volatile int *>(A.step_base) - A.it : A.it;
    const float *const img_ptr =
        A.step_base ? reinterpret_cast<const float *>(reinterpret_cast<const char *>(A.img_base) +
                                                      (long long)(it - A.img_t0) * A.img_step *
                                                          (img_fmt == kImgBF16 ? 2 : img_fmt == kImgF24 ? 3 : 4))
                    : A.img;
    const bool fast = A.tile_fast[tile] != 0;
    const int rcv0 = A.rcv_ptr[tile], rcv1 = A.rcv_ptr[tile + 1];
    const bool has_rcv = rcv1 > rcv0 && (A.res_p || A.res_vx || A.res_vz);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(&bars[2], SM::COEF_BYTES);
        tma_load_2d(sA1, mA1, &bars[2], x0 - 4, z0 - R);
        tma_load_2d(sA2, mA2, &bars[2], x0 - 4, z0);
        for (int k = 0; k < 2 && k < ns; ++k)
            stage_loads<R>(mP, mVX, mVZ, smem + k * G::STAGE_FL, &bars[k], G::STAGE_BYTES, x0, z0, s0 + k,
                           G::P_FL, G::VX_FL);
    }
    if (!__syncthreads_and(mbar_wait_bounded(&bars[2], 0))) {
        if (threadIdx.x == 0) {
            atomicExch(A.err, -4);
            for (int k = 0; k < 2 && k < ns; ++k) mbar_wait_bounded(&bars[k], 0);
        }
        return;
    }

    const int gx0 = x0 - 4 + 4 * lane;
    const int rb = warp * G::LP, rc = min(G::LP, G::PR - rb);
    const int vb = warp * G::LV, vcnt = min(G::LV, TZ - vb);
    const bool vlane = lane >= 1 && lane <= 30;

    // per-thread partial sums over this CTA's shots (tile cells)
    float4 acc1[G::LV], acc2[G::LV];
#pragma unroll
    for (int u = 0; u < G::LV; ++u) {
        acc1[u] = zero4();
        acc2[u] = zero4();
    }

    for (int k = 0; k < ns; ++k) {
        const int s = s0 + k;
        const int b = k & 1;
        // imaging fields of this shot's tile cells: issued now, used in stage B
        ImgRaw im[G::LV], jx[G::LV], jz[G::LV];
#pragma unroll
        for (int u = 0; u < G::LV; ++u) {
            const int gz = z0 + vb + u;
            const bool ok = vlane && u < vcnt && gz < g.Nz && gx0 < g.Nx;
            const long long io = (long long)s * g.plane + (long long)gz * g.pitch + gx0;
            im[u] = ok ? load_img_raw(img_ptr, io, img_fmt) : img_raw_zero();
            if (RHO) {
                jx[u] = ok ? load_img_raw(img_ptr, io + A.img_field_stride, img_fmt) : img_raw_zero();
                jz[u] = ok ? load_img_raw(img_ptr, io + 2 * A.img_field_stride, img_fmt) : img_raw_zero();
            }
        }
        // every thread waits (bounded) for this shot's stage; no CTA barrier
        // here: the refill of shot k-1's buffer waits for the mid-shot
        // barrier below, which every thread reaches only after finishing
        // shot k-1.  A give-up sets the status word and the launch runs on
        // (every thread still meets every barrier); its results are void.
        if (!mbar_wait_bounded(&bars[b], (k >> 1) & 1)) atomicExch(A.err, -4);
        float *sP = smem + b * G::STAGE_FL;
        float *sVX = sP + G::P_FL;
        float *sVZ = sVX + G::VX_FL;

        // ---------------- adjoint sources at the receivers ------------------
        if (has_rcv) {
            for (int e = rcv0 + threadIdx.x; e < rcv1; e += NTHR) {
                const int4 en = A.rcv_ent[e];
                const int gz = en.x, gx = en.y;
                const long long t = ((long long)s * g.nt + it) * g.n_rcv + en.z;
                const long long o = (long long)gz * g.pitch + gx;
                // a receiver in the mirror row fs-1 records p[fs-1] = -p[fs+1]
                // and vz[fs-1] = vz[fs] (acoustic_2d.py:240-241, 268-274):
                // its adjoint sources go to those rows
                const bool mir = FS && gz == g.fs - 1;
                const int zp = mir ? g.fs + 1 : gz, zv = mir ? g.fs : gz;
                if (A.res_p && zp >= g.p_r0 && zp <= g.p_r1 && gx >= g.p_c0 && gx <= g.p_c1) {
                    const int r = zp - (z0 - R), c = gx - (x0 - 4);
                    const long long op = (long long)zp * g.pitch + gx;
                    const float src = A.a1[op] * A.res_p[t];
                    if (r >= 0 && r < G::PR && c >= 0 && c < RW) atomicAdd(&sP[r * RW + c], mir ? -src : src);
                }
                if (A.res_vx && gz >= g.vx_r0 && gz <= g.vx_r1 && gx >= g.vx_c0 && gx <= g.vx_c1) {
                    const int r = gz - (z0 - R), c = gx - (x0 - 8);
                    if (r >= 0 && r < G::PR && c >= 0 && c < VXW)
                        atomicAdd(&sVX[r * VXW + c], A.a2[o] * A.res_vx[t]);
                }
                if (A.res_vz && zv >= g.vz_r0 && zv <= g.vz_r1 && gx >= g.vz_c0 && gx <= g.vz_c1) {
                    const int r = zv - (z0 - 2 * R), c = gx - (x0 - 4);
                    if (r >= 0 && r < G::ZR && c >= 0 && c < RW)
                        atomicAdd(&sVZ[r * RW + c], A.a2[(long long)zv * g.pitch + gx] * A.res_vz[t]);
                }
            }
            __syncthreads();
        }

        // ---------------- stage A: mu_p on the whole sP rectangle ----------
        {
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
                    const float4 a1 = lds4(sA1 + r * RW + 4 * lane);
                    float D[4];
                    if (fast) {
                        divergence4<R>(sVX + r * VXW, lane, wz, u, g.c, D);
#pragma unroll
                        for (int q = 0; q < 4; ++q) at(pv, q) = __fmaf_rn(at(a1, q), D[q], at(pv, q));
                    } else {
                        const bool row_in = gz >= g.p_r0 && gz <= g.p_r1;
                        if (row_in && (gx0 + 3 >= g.p_c0) && (gx0 <= g.p_c1)) {
                            divergence4<R>(sVX + r * VXW, lane, wz, u, g.c, D);
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                float d = D[q];
                                if (FS && gz == g.fs + 1) {
                                    // share of the mirror row p[fs-1] = -p[fs+1]
                                    float M = 0.f;
#pragma unroll
                                    for (int kk = 0; kk < R; ++kk) M = __fmaf_rn(g.c[kk], at(wz[u + R - 2 + kk], q), M);
                                    d -= M;
                                }
                                const int gx = gx0 + q;
                                at(pv, q) = (gx >= g.p_c0 && gx <= g.p_c1) ? __fmaf_rn(at(a1, q), d, at(pv, q)) : 0.f;
                            }
                        } else {
                            pv = zero4();
                        }
                    }
                    sts4(sP + r * RW + 4 * lane, pv);
                }
            }
        }
        __syncthreads();
        // every thread is done with shot k-1: refill its buffer with shot k+1
        // (its generic-proxy writes were fenced at the end of shot k-1)
        if (threadIdx.x == 0 && k >= 1 && k + 1 < ns)
            stage_loads<R>(mP, mVX, mVZ, smem + (b ^ 1) * G::STAGE_FL, &bars[b ^ 1], G::STAGE_BYTES, x0, z0,
                           s + 1, G::P_FL, G::VX_FL);
        if (A.grad_wavelet && threadIdx.x == 0) {
            // the tile that owns the source cell: mu_p / a1 there is lambda_p
            const int sz = A.src_z[s], sx = A.src_x[s];
            if (sz >= z0 && sz < z0 + TZ && sx >= x0 && sx < x0 + TX) {
                const int r = sz - (z0 - R), c = sx - (x0 - 4);
                A.grad_wavelet[(long long)s * g.nt + it] = g.dt * (sP[r * RW + c] / sA1[r * RW + c]);
            }
        }

        // ---------------- stage B: tile --------------------------------------
        if (vlane) {
            float4 wp[G::LV + 2 * R - 1];
#pragma unroll
            for (int t = 0; t < G::LV + 2 * R - 1; ++t)
                wp[t] = (t < vcnt + 2 * R - 1) ? lds4(sP + (vb + 1 + t) * RW + 4 * lane) : zero4();
#pragma unroll
            for (int u = 0; u < G::LV; ++u) {
                if (u < vcnt) {
                    const int rv = vb + u;
                    const int rr = rv + R;
                    const int gz = z0 + rv;
                    if (fast || (gz < g.Nz && gx0 < g.Nx)) {
                        float Dx[4], Dz[4];
                        float4 mp1;
                        grad_x4<R>(sP + rr * RW, lane, g.c, Dx, mp1);
                        grad_z4<R>(wp, u, g.c, Dz);
                        const float4 vx1 = lds4(sVX + rr * VXW + 4 * lane + 4);
                        const float4 vz1 = lds4(sVZ + (rv + 2 * R) * RW + 4 * lane);
                        const float4 a2 = lds4(sA2 + rv * RW + 4 * lane);
                        const long long o = (long long)gz * g.pitch + gx0;
                        const float4 imv = decode_img4(im[u], img_fmt);
                        const float4 jxv = RHO ? decode_img4(jx[u], img_fmt) : zero4();
                        const float4 jzv = RHO ? decode_img4(jz[u], img_fmt) : zero4();
                        float4 vx, vz, pp;
                        if (fast) {
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                at(vx, q) = __fmaf_rn(at(a2, q), Dx[q], at(vx1, q));
                                at(vz, q) = __fmaf_rn(at(a2, q), Dz[q], at(vz1, q));
                                at(acc1[u], q) = __fmaf_rn(at(mp1, q), at(imv, q), at(acc1[u], q));
                            }
                            pp = mp1;
                            if (RHO) {
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    at(acc2[u], q) = __fmaf_rn(at(vx1, q), at(jxv, q), at(acc2[u], q));
                                    at(acc2[u], q) = __fmaf_rn(at(vz1, q), at(jzv, q), at(acc2[u], q));
                                }
                            }
                        } else {
                            vx = zero4(); vz = zero4(); pp = zero4();
                            const bool vx_row = gz >= g.vx_r0 && gz <= g.vx_r1;
                            const bool vz_row = gz >= g.vz_r0 && gz <= g.vz_r1;
                            const bool p_row = gz >= g.p_r0 && gz <= g.p_r1;
                            const bool any_v = (vx_row && gx0 + 3 >= g.vx_c0 && gx0 <= g.vx_c1) ||
                                               (vz_row && gx0 + 3 >= g.vz_c0 && gx0 <= g.vz_c1);
                            const bool any_p = p_row && gx0 + 3 >= g.p_c0 && gx0 <= g.p_c1;
                            if (any_v) {
                                const float4 k2 = ldg4(A.k2 + o);
                                const float4 k3 = ldg4(A.k3 + o);
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    const int gx = gx0 + q;
                                    if (vx_row && gx >= g.vx_c0 && gx <= g.vx_c1) {
                                        at(vx, q) = __fmaf_rn(at(a2, q), Dx[q], (1.f - at(k2, q)) * at(vx1, q));
                                        if (RHO) at(acc2[u], q) = __fmaf_rn(at(vx1, q), at(jxv, q), at(acc2[u], q));
                                    }
                                    if (vz_row && gx >= g.vz_c0 && gx <= g.vz_c1) {
                                        float d = Dz[q];
                                        if (FS && gz == g.fs) {
                                            // the p update reads vz[fs-1] as vz[fs]
#pragma unroll
                                            for (int kk = 0; kk < R; ++kk) d = __fmaf_rn(g.c[kk], at(wp[u + R - 1 + kk], q), d);
                                        }
                                        at(vz, q) = __fmaf_rn(at(a2, q), d, (1.f - at(k3, q)) * at(vz1, q));
                                        if (RHO) at(acc2[u], q) = __fmaf_rn(at(vz1, q), at(jzv, q), at(acc2[u], q));
                                    }
                                }
                            }
                            if (any_p) {
                                const float4 k1 = ldg4(A.k1 + o);
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    const int gx = gx0 + q;
                                    if (gx >= g.p_c0 && gx <= g.p_c1) {
                                        at(pp, q) = (1.f - at(k1, q)) * at(mp1, q);
                                        at(acc1[u], q) = __fmaf_rn(at(mp1, q), at(imv, q), at(acc1[u], q));
                                    }
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
        // order this shot's generic-proxy shared-memory writes before the TMA
        // that refills the buffer (after the next shot's mid-shot barrier)
        fence_proxy_async_smem();
    }

    // compensated accumulation of this step's partial sums into the group's
    // running totals (this CTA is their only writer for this tile)
    if (vlane) {
#pragma unroll
        for (int u = 0; u < G::LV; ++u) {
            const int gz = z0 + vb + u;
            if (u < vcnt && gz >= g.p_r0 && gz <= g.p_r1 && gx0 < g.Nx) {
                const long long o = (long long)group * g.plane + (long long)gz * g.pitch + gx0;
                float4 s1 = *reinterpret_cast<float4 *>(A.G1 + o), c1 = *reinterpret_cast<float4 *>(A.C1 + o);
#pragma unroll
                for (int q = 0; q < 4; ++q) neumaier_add(at(s1, q), at(c1, q), at(acc1[u], q));
                stg4(A.G1 + o, s1);
                stg4(A.C1 + o, c1);
            }
            if (RHO && u < vcnt && gz < g.Nz && gx0 < g.Nx) {
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

template <int R, int TZ, bool FS, bool RHO, int IMGF>
__global__ void __launch_bounds__(NTHR, TZ <= 16 ? 2 : 1)
adj_step_kernel(const __grid_constant__ CUtensorMap mP, const __grid_constant__ CUtensorMap mVX,
                const __grid_constant__ CUtensorMap mVZ, const __grid_constant__ CUtensorMap mA1,
                const __grid_constant__ CUtensorMap mA2, const AdjArgs A)
{
    const int group = A.grp0 + (int)(blockIdx.x % A.grp_count);
    const int rank = (int)(blockIdx.x / A.grp_count);
    const int tile = A.tile_order ? A.tile_order[rank] : rank;
    adj_body<R, TZ, FS, RHO, IMGF>(&mP, &mVX, &mVZ, &mA1, &mA2, A, group, tile);
}

template <int R, int TZ>
constexpr size_t adj_smem_bytes()
{
    return StepSmem<R, TZ>::BYTES;
}

// dL/dvp and dL/drho on the (nz, nx) model: per padded cell
//   G1 = sum(mu_p1 * I), G2 = sum(mu_v1 * J) over groups (compensated),
//   dL/dc = 2 G1 / c, dL/dden = (G1 + G2) / den,
// then the adjoint of pad_model: each model cell collects every padded cell
// it was replicated into (acoustic_2d.py:55-64).  Internal linkage: the
// translation units that instantiate the step kernels include this header too.
static __global__ void grad_finish_kernel(const float *__restrict__ vp, const float *__restrict__ rho,
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
