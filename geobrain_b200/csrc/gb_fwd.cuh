// Fused forward time step of the 2D acoustic staggered-grid scheme.
//
// One launch advances every shot of one model by one time step:
//   p  <- (1 - k1) p - a1 * div(vx, vz)          on the p mask  (ref :211-226)
//   p  += dt * wavelet[s, it]   at the source                    (ref :228-237)
//   p[fs-1] = -p[fs+1]          free surface, in shared memory   (ref :240-241)
//   vx <- (1 - k2) vx - a2 * dx(p)               on the vx mask  (ref :244-253)
//   vz <- (1 - k3) vz - a2 * dz(p)               on the vz mask  (ref :256-265)
//   vz[fs-1] = vz[fs]           free surface, applied on load    (ref :268-269)
//   traces[s, it, r] = (p, vx, vz)[receiver r]                   (ref :272-274)
//   energy += sum_s (p^2, vx^2, vz^2) over the interior          (ref :277-285)
// ("ref" = geobrain/physics/wave/kernels/acoustic_2d.py.)
//
// The two free-surface mirror rows are never stored: row fs-1 of p and vz is
// only ever read by the next stage, so each CTA rebuilds it in shared memory
// from the rows it mirrors.  Every other cell follows the reference exactly.
#pragma once

#include "gb_device.cuh"

namespace gb {

struct StepGeom {
    int Nz, Nx, pitch;
    int nz, nx, pml, fs;
    int p_r0, p_r1, p_c0, p_c1;
    int vx_r0, vx_r1, vx_c0, vx_c1;
    int vz_r0, vz_r1, vz_c0, vz_c1;
    int tiles_x, n_tiles;
    int n_shots, shots_per_cta, n_groups;
    int nt, n_rcv;
    float dt;
    float c[4];
    long long plane;   // Nz * pitch
};

struct FwdArgs {
    StepGeom g;
    int it;                          // time step index
    const float *a1, *k1, *a2, *k2, *k3;   // coefficient planes, Nz x pitch
    float *out;                      // next state [S][3][plane]
    const int *src_z, *src_x;        // padded source cells
    const float *wavelet;            // [S][nt]
    const int *rcv_ptr;              // CSR over tiles
    const int4 *rcv_ent;             // (row in tile, col in tile, receiver, 0)
    float *tr_p, *tr_vx, *tr_vz;     // [S][nt][n_rcv] or null
    float *energy;                   // [3][plane] padded accumulators or null
    float *imaging;                  // [S][plane] -div(v) on the p mask, or null
    long long img_field_stride;      // IMG == 2: dx(p), dz(p) blocks follow at this stride
    int *err;
};

template <int R>
__device__ __forceinline__ void stage_loads(const CUtensorMap *mP, const CUtensorMap *mVX, const CUtensorMap *mVZ,
                                            float *buf, uint64_t *bar, uint32_t bytes, int x0, int z0,
                                            int s, int P_FL, int VX_FL)
{
    mbar_arrive_expect_tx(bar, bytes);
    tma_load_3d(buf, mP, bar, x0 - 4, z0 - R, 3 * s + 0);
    tma_load_3d(buf + P_FL, mVX, bar, x0 - 8, z0 - R, 3 * s + 1);
    tma_load_3d(buf + P_FL + VX_FL, mVZ, bar, x0 - 4, z0 - 2 * R, 3 * s + 2);
}

// IMG: 0 no imaging fields; 1 store I = -div(v^n) on the p mask (velocity
// gradient); 2 also store Jx = dx(p), Jz = dz(p) on the vx / vz masks (density).
template <int R, int TZ, bool FS, bool ENERGY, int IMG>
__global__ void __launch_bounds__(NTHR, 1)
fwd_step_kernel(const __grid_constant__ CUtensorMap mP, const __grid_constant__ CUtensorMap mVX,
                const __grid_constant__ CUtensorMap mVZ, const FwdArgs A)
{
    using G = Geo<R, TZ>;
    const StepGeom &g = A.g;
    extern __shared__ __align__(128) float smem[];
    float *stage[2] = {smem, smem + G::STAGE_FL};
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * G::STAGE_FL);
    float *eacc = reinterpret_cast<float *>(bars + 2);   // [3][TZ][TX] when ENERGY

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
    if (ENERGY) {
        for (int i = threadIdx.x; i < 3 * TZ * TX; i += NTHR) eacc[i] = 0.f;
    }

    // this thread's columns in the 128-wide rectangles: x0 - 4 + 4*lane + q
    const int gx0 = x0 - 4 + 4 * lane;

    for (int k = 0; k < ns; ++k) {
        const int s = s0 + k;
        const int b = k & 1;
        // every thread polls (bounded); the vote makes the give-up decision
        // uniform so no thread is left waiting at a barrier
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

        if (FS) {
            // vz[fs-1] = vz[fs]: rebuild the mirror row the previous step did not store
            const int rm = g.fs - 1 - (z0 - 2 * R);
            if (rm >= 0 && rm + 1 < G::ZR)
                for (int c = threadIdx.x; c < RW; c += NTHR) sVZ[rm * RW + c] = sVZ[(rm + 1) * RW + c];
            __syncthreads();
        }

        // ---------------- p-stage: whole sP rectangle, in place -------------
        {
            const int rb = warp * G::LP;
            const int rc = min(G::LP, G::PR - rb);
            float4 wz[G::LP + 2 * R - 1];
#pragma unroll
            for (int t = 0; t < G::LP + 2 * R - 1; ++t)
                wz[t] = (t < rc + 2 * R - 1) ? lds4(sVZ + (rb + t) * RW + 4 * lane) : zero4();
            const int sz = A.src_z[s], sx = A.src_x[s];
#pragma unroll
            for (int u = 0; u < G::LP; ++u) {
                if (u < rc) {
                    const int r = rb + u;
                    const int gz = z0 - R + r;
                    float e[12];
                    {
                        const float4 e0 = lds4(sVX + r * VXW + 4 * lane);
                        const float4 e1 = lds4(sVX + r * VXW + 4 * lane + 4);
                        const float4 e2 = lds4(sVX + r * VXW + 4 * lane + 8);
                        e[0] = e0.x; e[1] = e0.y; e[2] = e0.z; e[3] = e0.w;
                        e[4] = e1.x; e[5] = e1.y; e[6] = e1.z; e[7] = e1.w;
                        e[8] = e2.x; e[9] = e2.y; e[10] = e2.z; e[11] = e2.w;
                    }
                    float4 pv = lds4(sP + r * RW + 4 * lane);
                    const bool row_in = gz >= g.p_r0 && gz <= g.p_r1;
                    const bool unit_in = row_in && (gx0 + 3 >= g.p_c0) && (gx0 <= g.p_c1);
                    if (unit_in) {
                        const long long o = (long long)gz * g.pitch + gx0;
                        const float4 a1 = ldg4(A.a1 + o);
                        const float4 k1 = ldg4(A.k1 + o);
                        float4 img;
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            float D = 0.f;
#pragma unroll
                            for (int kk = 0; kk < R; ++kk)
                                D += g.c[kk] * (((e[q + 4 + kk] - e[q + 3 - kk]) + at(wz[u + R + kk], q)) -
                                                at(wz[u + R - 1 - kk], q));
                            const int gx = gx0 + q;
                            const bool m = gx >= g.p_c0 && gx <= g.p_c1;
                            at(img, q) = m ? -D : 0.f;
                            if (m) at(pv, q) = (1.f - at(k1, q)) * at(pv, q) - at(a1, q) * D;
                        }
                        if (IMG >= 1 && r >= R && r < R + TZ && lane >= 1 && lane <= 30)
                            stg4(A.imaging + (long long)s * g.plane + o, img);
                    }
                    if (gz == sz && sx >= gx0 && sx < gx0 + 4)
                        at(pv, sx - gx0) += g.dt * A.wavelet[(long long)s * g.nt + A.it];
                    sts4(sP + r * RW + 4 * lane, pv);
                }
            }
        }
        __syncthreads();

        if (FS) {
            // p[fs-1] = -p[fs+1] inside the rectangle
            const int rm = g.fs - 1 - (z0 - R);
            if (rm >= 0 && rm + 2 < G::PR)
                for (int c = threadIdx.x; c < RW; c += NTHR) sP[rm * RW + c] = -sP[(rm + 2) * RW + c];
            __syncthreads();
        }

        // ---------------- v-stage: tile only -------------------------------
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
                    const int rv = vb + u;          // tile row
                    const int rr = rv + R;          // sP / sVX row
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
                        float4 vx = lds4(sVX + rr * VXW + 4 * lane + 4);
                        float4 vz = lds4(sVZ + (rv + 2 * R) * RW + 4 * lane);
                        const long long o = (long long)gz * g.pitch + gx0;
                        const bool vx_row = gz >= g.vx_r0 && gz <= g.vx_r1;
                        const bool vz_row = gz >= g.vz_r0 && gz <= g.vz_r1;
                        const bool need = (vx_row && gx0 + 3 >= g.vx_c0 && gx0 <= g.vx_c1) ||
                                          (vz_row && gx0 + 3 >= g.vz_c0 && gx0 <= g.vz_c1);
                        float4 jx = zero4(), jz = zero4();
                        if (need) {
                            const float4 a2 = ldg4(A.a2 + o);
                            const float4 k2 = ldg4(A.k2 + o);
                            const float4 k3 = ldg4(A.k3 + o);
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const int gx = gx0 + q;
                                if (vx_row && gx >= g.vx_c0 && gx <= g.vx_c1) {
                                    float D = 0.f;
#pragma unroll
                                    for (int kk = 0; kk < R; ++kk)
                                        D += g.c[kk] * (f[q + 5 + kk] - f[q + 4 - kk]);
                                    at(vx, q) = (1.f - at(k2, q)) * at(vx, q) - at(a2, q) * D;
                                    at(jx, q) = D;
                                }
                                if (vz_row && gx >= g.vz_c0 && gx <= g.vz_c1) {
                                    float D = 0.f;
#pragma unroll
                                    for (int kk = 0; kk < R; ++kk)
                                        D += g.c[kk] * (at(wp[u + R + kk], q) - at(wp[u + R - 1 - kk], q));
                                    at(vz, q) = (1.f - at(k3, q)) * at(vz, q) - at(a2, q) * D;
                                    at(jz, q) = D;
                                }
                            }
                        }
                        if (IMG == 2) {
                            stg4(A.imaging + (long long)s * g.plane + A.img_field_stride + o, jx);
                            stg4(A.imaging + (long long)s * g.plane + 2 * A.img_field_stride + o, jz);
                        }
                        const float4 pv = make_float4(f[4], f[5], f[6], f[7]);
                        float *outs = A.out + (long long)s * 3 * g.plane + o;
                        stg4(outs, pv);
                        stg4(outs + g.plane, vx);
                        stg4(outs + 2 * g.plane, vz);
                        sts4(sVX + rr * VXW + 4 * lane + 4, vx);
                        sts4(sVZ + (rv + 2 * R) * RW + 4 * lane, vz);
                        if (ENERGY && gz >= g.pml && gz < g.pml + g.nz) {
                            float *ea = eacc + rv * TX + 4 * (lane - 1);
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const int gx = gx0 + q;
                                if (gx >= g.pml && gx < g.pml + g.nx) {
                                    ea[q] += at(pv, q) * at(pv, q);
                                    ea[TZ * TX + q] += at(vx, q) * at(vx, q);
                                    ea[2 * TZ * TX + q] += at(vz, q) * at(vz, q);
                                }
                            }
                        }
                    }
                }
            }
        }
        __syncthreads();

        // ---------------- receivers of this tile ---------------------------
        if (A.tr_p || A.tr_vx || A.tr_vz) {
            const int e0 = A.rcv_ptr[tile], e1 = A.rcv_ptr[tile + 1];
            for (int e = e0 + threadIdx.x; e < e1; e += NTHR) {
                const int4 en = A.rcv_ent[e];
                const int rr = en.x + R, cc = en.y + 4;
                const long long t = ((long long)s * g.nt + A.it) * g.n_rcv + en.z;
                if (A.tr_p) A.tr_p[t] = sP[rr * RW + cc];
                if (A.tr_vx) A.tr_vx[t] = sVX[rr * VXW + cc + 4];
                if (A.tr_vz) A.tr_vz[t] = sVZ[(en.x + 2 * R) * RW + cc];
            }
        }
        // order this iteration's generic-proxy shared-memory writes before the
        // TMA that refills the buffer
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0 && k + 2 < ns) {
            stage_loads<R>(&mP, &mVX, &mVZ, stage[b], &bars[b], G::STAGE_BYTES, x0, z0, s + 2, G::P_FL,
                           G::VX_FL);
        }
    }

    if (ENERGY) {
        // add this CTA's partial sums (over its shots) into the padded maps
        for (int i = threadIdx.x; i < TZ * (TX / 4); i += NTHR) {
            const int rv = i / (TX / 4), c4 = i % (TX / 4);
            const int gz = z0 + rv, gx = x0 + 4 * c4;
            if (gz < g.Nz && gx < g.Nx) {
                const long long o = (long long)gz * g.pitch + gx;
#pragma unroll
                for (int f = 0; f < 3; ++f)
                    red_add_v4(A.energy + f * g.plane + o, lds4(eacc + f * TZ * TX + rv * TX + 4 * c4));
            }
        }
    }
}

template <int R, int TZ, bool ENERGY>
constexpr size_t fwd_smem_bytes()
{
    return 2 * Geo<R, TZ>::STAGE_BYTES + 16 + (ENERGY ? 3 * TZ * TX * 4 : 0);
}

}  // namespace gb
