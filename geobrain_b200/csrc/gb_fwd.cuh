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
//
// Tiles whose halo rectangles lie inside every update mask and see no
// damping (most of the grid: the PML is a thin frame) take a fast path with
// no per-cell masks and no damping terms; the arithmetic of the cells is the
// same either way.
#pragma once

#include "gb_stencil.cuh"

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
    int it;                          // time step index (offset from *step_base when that is set)
    const int *step_base;            // device step counter of a graph-replayed chunk, or null
    const float *a1, *k1, *a2, *k2, *k3;   // coefficient planes, Nz x pitch
    const int *tile_fast;            // per tile: 1 = no masks and no damping anywhere it reads
    float *out;                      // next state [S][3][plane]
    const int *src_z, *src_x;        // padded source cells
    const float *wavelet;            // [S][nt]
    const int *rcv_ptr;              // CSR over tiles
    const int4 *rcv_ent;             // (row in tile, col in tile, receiver, 1: p and vx / 2: vz / 3: all)
    float *tr_p, *tr_vx, *tr_vz;     // [S][nt][n_rcv] or null
    float *energy;                   // [3][plane] padded accumulators or null
    float *imaging;                  // [S][plane] -div(v) on the p mask, or null
    long long img_field_stride;      // IMG == 2: dx(p), dz(p) blocks follow at this stride (elements)
    int img_fmt;                     // storage format of the imaging fields (kImg*)
    // graph replay (step_base set): the imaging fields of step it are at
    // img_base + (it - img_t0) * img_step elements, when img_base is set
    float *img_base;
    long long img_step;
    int img_t0;
    int grp0, grp_count;             // shot groups this launch covers
    // the launch's work list: CTA b does shots [y, y + z) of tile x of
    // items[b]; null: CTA b does group grp0 + b % grp_count of tile b / grp_count
    const int4 *items;
    int *err;
    // CPML option (null otherwise): profiles [bz, az (integer rows), bz, az
    // (half rows)][Nz] then [bx, ax (integer cols), bx, ax (half cols)][pitch],
    // and the memory variables [S][psi_px, psi_pz, psi_vx, psi_vz][plane],
    // read from psi_in and written to psi_out (two levels, as the state)
    const float *cpml;
    const float *psi_in;
    float *psi_out;
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

// Shared-memory layout of both step kernels: two field stages, then a1 on
// the p rectangle and a2 on the tile rows (loaded once per CTA), then the
// mbarriers.
template <int R, int TZ>
struct StepSmem {
    using G = Geo<R, TZ>;
    static constexpr int A1_FL = G::PR * RW;
    static constexpr int A2_FL = TZ * RW;
    static constexpr int COEF_FL = A1_FL + A2_FL;
    static constexpr uint32_t COEF_BYTES = COEF_FL * 4u;
    static constexpr size_t BYTES = 2 * G::STAGE_BYTES + COEF_BYTES + 32;
};

// Does this tile need per-cell masks?  (Pure geometry; the damping part of
// the fast-path test is precomputed per tile in tile_fast.)
template <int R, int TZ>
__device__ __forceinline__ bool tile_is_interior(const StepGeom &g, int z0, int x0)
{
    return z0 - 2 * R >= g.fs + 1 && z0 - R >= g.p_r0 && z0 + TZ + R - 1 <= g.p_r1 && x0 - 4 >= g.p_c0 &&
           x0 + TX + 3 <= g.p_c1 && z0 >= g.vx_r0 && z0 >= g.vz_r0 && z0 + TZ - 1 <= g.vx_r1 &&
           z0 + TZ - 1 <= g.vz_r1 && x0 >= g.vx_c0 && x0 >= g.vz_c0 && x0 + TX - 1 <= g.vx_c1 &&
           x0 + TX - 1 <= g.vz_c1;
}

// IMG: 0 no imaging fields; 1 store I = -div(v^n) on the p mask (velocity
// gradient); 2 also store Jx = dx(p), Jz = dz(p) on the vx / vz masks (density).
// The body of one CTA: shots [s0, s0 + ns) (ns <= kMaxShotsPerCta) of tile
// `tile` of the model A describes; the maps are the TMA descriptors of the
// input state and of the a1 / a2 planes.
template <int R, int TZ, bool FS, bool ENERGY, int IMG>
__device__ __forceinline__ void fwd_body(const CUtensorMap *mP, const CUtensorMap *mVX, const CUtensorMap *mVZ,
                                         const CUtensorMap *mA1, const CUtensorMap *mA2,
                                         const FwdArgs &__restrict__ A, const int tile, const int s0, const int ns)
{
    using G = Geo<R, TZ>;
    using SM = StepSmem<R, TZ>;
    const StepGeom &__restrict__ g = A.g;
    extern __shared__ __align__(128) float smem[];
    __shared__ int2 s_src[kMaxShotsPerCta];   // (z, x) source cell of each shot of this CTA
    float *sA1 = smem + 2 * G::STAGE_FL;
    float *sA2 = sA1 + SM::A1_FL;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sA1 + SM::COEF_FL);

    const int z0 = (tile / g.tiles_x) * TZ;
    const int x0 = (tile % g.tiles_x) * TX;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1);
        fence_mbar_init();
    }
    grid_dependency_wait();
    grid_launch_dependents();
    // a CUDA graph replays the same launches for every chunk of steps; the
    // chunk's first step comes from device memory
    const int it = A.step_base ? *reinterpret_cast<const volatile int *>(A.step_base) + A.it : A.it;
    float *const imaging = A.step_base && A.img_base
                               ? reinterpret_cast<float *>(reinterpret_cast<char *>(A.img_base) +
                                                           (long long)(it - A.img_t0) * A.img_step *
                                                               (A.img_fmt == kImgBF16 ? 2 : A.img_fmt == kImgF24 ? 3 : 4))
                               : A.imaging;
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(&bars[2], SM::COEF_BYTES);
        tma_load_2d(sA1, mA1, &bars[2], x0 - 4, z0 - R);
        tma_load_2d(sA2, mA2, &bars[2], x0 - 4, z0);
        for (int k = 0; k < 2 && k < ns; ++k)
            stage_loads<R>(mP, mVX, mVZ, smem + k * G::STAGE_FL, &bars[k], G::STAGE_BYTES, x0, z0, s0 + k,
                           G::P_FL, G::VX_FL);
    }
    for (int k = threadIdx.x; k < ns; k += NTHR) s_src[k] = make_int2(A.src_z[s0 + k], A.src_x[s0 + k]);
    const bool fast = A.tile_fast[tile] != 0;
    const int rcv0 = A.rcv_ptr[tile], rcv1 = A.rcv_ptr[tile + 1];
    const bool has_rcv = rcv1 > rcv0 && (A.tr_p || A.tr_vx || A.tr_vz);
    if (!__syncthreads_and(mbar_wait_bounded(&bars[2], 0))) {
        if (threadIdx.x == 0) {
            atomicExch(A.err, -4);
            for (int k = 0; k < 2 && k < ns; ++k) mbar_wait_bounded(&bars[k], 0);
        }
        return;
    }

    const int gx0 = x0 - 4 + 4 * lane;   // first of this thread's 4 columns
    const int rb = warp * G::LP, rc = min(G::LP, G::PR - rb);      // p-stage rows of this warp
    const int vb = warp * G::LV, vcnt = min(G::LV, TZ - vb);       // v-stage rows of this warp
    const bool vlane = lane >= 1 && lane <= 30;

    float4 e_p[G::LV], e_vx[G::LV], e_vz[G::LV];
    if (ENERGY) {
#pragma unroll
        for (int u = 0; u < G::LV; ++u) e_p[u] = e_vx[u] = e_vz[u] = zero4();
    }

    for (int k = 0; k < ns; ++k) {
        const int s = s0 + k;
        const int b = k & 1;
        // every thread waits (bounded) for this shot's stage; no CTA barrier
        // here: the refill of shot k-1's buffer waits for the mid-shot
        // barrier below, which every thread reaches only after finishing
        // shot k-1.  A give-up sets the status word and the launch runs on
        // (every thread still meets every barrier); its results are void.
        if (!mbar_wait_bounded(&bars[b], (k >> 1) & 1)) atomicExch(A.err, -4);
        float *sP = smem + b * G::STAGE_FL;
        float *sVX = sP + G::P_FL;
        float *sVZ = sVX + G::VX_FL;

        if (FS && !fast) {
            // vz[fs-1] = vz[fs]: rebuild the mirror row the previous step did not store
            const int rm = g.fs - 1 - (z0 - 2 * R);
            if (rm >= 0 && rm + 1 < G::ZR)
                for (int c = threadIdx.x; c < RW; c += NTHR) sVZ[rm * RW + c] = sVZ[(rm + 1) * RW + c];
            __syncthreads();
        }

        // ---------------- p-stage: whole sP rectangle, in place -------------
        {
            float4 wz[G::LP + 2 * R - 1];
#pragma unroll
            for (int t = 0; t < G::LP + 2 * R - 1; ++t)
                wz[t] = (t < rc + 2 * R - 1) ? lds4(sVZ + (rb + t) * RW + 4 * lane) : zero4();
            const int2 src = s_src[k];
            const int sz = src.x, sx = src.y;
#pragma unroll
            for (int u = 0; u < G::LP; ++u) {
                if (u < rc) {
                    const int r = rb + u;
                    const int gz = z0 - R + r;
                    float4 pv = lds4(sP + r * RW + 4 * lane);
                    float D[4];
                    const float4 a1 = lds4(sA1 + r * RW + 4 * lane);
                    const bool tile_cell = IMG >= 1 && r >= R && r < R + TZ && vlane;
                    if (fast) {
                        divergence4<R>(sVX + r * VXW, lane, wz, u, g.c, D);
#pragma unroll
                        for (int q = 0; q < 4; ++q) at(pv, q) = __fmaf_rn(-at(a1, q), D[q], at(pv, q));
                        if (tile_cell && imaging)
                            store_img4(imaging, (long long)s * g.plane + (long long)gz * g.pitch + gx0,
                                       A.img_fmt, make_float4(-D[0], -D[1], -D[2], -D[3]));
                    } else {
                        const bool row_in = gz >= g.p_r0 && gz <= g.p_r1;
                        if (row_in && (gx0 + 3 >= g.p_c0) && (gx0 <= g.p_c1)) {
                            const long long o = (long long)gz * g.pitch + gx0;
                            float4 img;
                            if (A.cpml) {
                                // psi' = b psi + a d, p' = p - a1 ((Dx + psi_x') + (Dz + psi_z'))
                                float Dx[4], Dz[4];
                                divergence4_split<R>(sVX + r * VXW, lane, wz, u, g.c, Dx, Dz);
                                const float bz = A.cpml[gz], az = A.cpml[g.Nz + gz];
                                const float *xp = A.cpml + 4 * g.Nz;
                                const float4 bx = ldg4(xp + gx0), ax = ldg4(xp + g.pitch + gx0);
                                const long long po = (long long)s * 4 * g.plane + o;
                                const float4 ox = ldg4(A.psi_in + po), oz = ldg4(A.psi_in + po + g.plane);
                                float4 nx = ox, nz = oz;
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    const int gx = gx0 + q;
                                    const bool m = gx >= g.p_c0 && gx <= g.p_c1;
                                    at(img, q) = 0.f;
                                    if (m) {
                                        at(nx, q) = __fadd_rn(__fmul_rn(at(bx, q), at(ox, q)), __fmul_rn(at(ax, q), Dx[q]));
                                        at(nz, q) = __fadd_rn(__fmul_rn(bz, at(oz, q)), __fmul_rn(az, Dz[q]));
                                        const float sd = __fadd_rn(__fadd_rn(Dx[q], at(nx, q)), __fadd_rn(Dz[q], at(nz, q)));
                                        at(pv, q) = __fsub_rn(at(pv, q), __fmul_rn(at(a1, q), sd));
                                        at(img, q) = -sd;
                                    }
                                }
                                stg4(A.psi_out + po, nx);
                                stg4(A.psi_out + po + g.plane, nz);
                            } else {
                                divergence4<R>(sVX + r * VXW, lane, wz, u, g.c, D);
                                const float4 k1 = ldg4(A.k1 + o);
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    const int gx = gx0 + q;
                                    const bool m = gx >= g.p_c0 && gx <= g.p_c1;
                                    at(img, q) = m ? -D[q] : 0.f;
                                    if (m) at(pv, q) = __fmaf_rn(-at(a1, q), D[q], (1.f - at(k1, q)) * at(pv, q));
                                }
                            }
                            if (tile_cell && imaging)
                                store_img4(imaging, (long long)s * g.plane + o, A.img_fmt, img);
                        }
                    }
                    if (gz == sz && sx >= gx0 && sx < gx0 + 4) {
                        // p + dt * w, rounded after the product and after the
                        // sum as the reference does (acoustic_2d.py:230-233)
                        const float amp = __fmul_rn(g.dt, A.wavelet[(long long)s * g.nt + it]);
                        const int q = sx - gx0;
                        if (q == 0) pv.x = __fadd_rn(pv.x, amp);
                        else if (q == 1) pv.y = __fadd_rn(pv.y, amp);
                        else if (q == 2) pv.z = __fadd_rn(pv.z, amp);
                        else pv.w = __fadd_rn(pv.w, amp);
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

        if (FS && !fast) {
            // p[fs-1] = -p[fs+1] inside the rectangle
            const int rm = g.fs - 1 - (z0 - R);
            if (rm >= 0 && rm + 2 < G::PR)
                for (int c = threadIdx.x; c < RW; c += NTHR) sP[rm * RW + c] = -sP[(rm + 2) * RW + c];
            __syncthreads();
        }

        // ---------------- v-stage: tile only -------------------------------
        if (vlane) {
            float4 wp[G::LV + 2 * R - 1];
#pragma unroll
            for (int t = 0; t < G::LV + 2 * R - 1; ++t)
                wp[t] = (t < vcnt + 2 * R - 1) ? lds4(sP + (vb + 1 + t) * RW + 4 * lane) : zero4();
#pragma unroll
            for (int u = 0; u < G::LV; ++u) {
                if (u < vcnt) {
                    const int rv = vb + u;          // tile row
                    const int rr = rv + R;          // sP / sVX row
                    const int gz = z0 + rv;
                    if (fast || (gz < g.Nz && gx0 < g.Nx)) {
                        float Dx[4], Dz[4];
                        float4 pv;
                        grad_x4<R>(sP + rr * RW, lane, g.c, Dx, pv);
                        grad_z4<R>(wp, u, g.c, Dz);
                        float4 vx = lds4(sVX + rr * VXW + 4 * lane + 4);
                        float4 vz = lds4(sVZ + (rv + 2 * R) * RW + 4 * lane);
                        const float4 a2 = lds4(sA2 + rv * RW + 4 * lane);
                        const long long o = (long long)gz * g.pitch + gx0;
                        float4 jx = zero4(), jz = zero4();
                        if (fast) {
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                at(vx, q) = __fmaf_rn(-at(a2, q), Dx[q], at(vx, q));
                                at(vz, q) = __fmaf_rn(-at(a2, q), Dz[q], at(vz, q));
                            }
                            if (IMG == 2) {
                                jx = make_float4(Dx[0], Dx[1], Dx[2], Dx[3]);
                                jz = make_float4(Dz[0], Dz[1], Dz[2], Dz[3]);
                            }
                        } else {
                            const bool vx_row = gz >= g.vx_r0 && gz <= g.vx_r1;
                            const bool vz_row = gz >= g.vz_r0 && gz <= g.vz_r1;
                            const bool need = (vx_row && gx0 + 3 >= g.vx_c0 && gx0 <= g.vx_c1) ||
                                              (vz_row && gx0 + 3 >= g.vz_c0 && gx0 <= g.vz_c1);
                            if (need && A.cpml) {
                                // psi' = b psi + a G, v' = v - a2 (G + psi')
                                const float bz = A.cpml[2 * g.Nz + gz], az = A.cpml[3 * g.Nz + gz];
                                const float *xp = A.cpml + 4 * g.Nz;
                                const float4 bx = ldg4(xp + 2 * g.pitch + gx0), ax = ldg4(xp + 3 * g.pitch + gx0);
                                const long long po = (long long)s * 4 * g.plane + o;
                                const float4 ox = ldg4(A.psi_in + po + 2 * g.plane), oz = ldg4(A.psi_in + po + 3 * g.plane);
                                float4 nx = ox, nz = oz;
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    const int gx = gx0 + q;
                                    if (vx_row && gx >= g.vx_c0 && gx <= g.vx_c1) {
                                        at(nx, q) = __fadd_rn(__fmul_rn(at(bx, q), at(ox, q)), __fmul_rn(at(ax, q), Dx[q]));
                                        at(jx, q) = __fadd_rn(Dx[q], at(nx, q));
                                        at(vx, q) = __fsub_rn(at(vx, q), __fmul_rn(at(a2, q), at(jx, q)));
                                    }
                                    if (vz_row && gx >= g.vz_c0 && gx <= g.vz_c1) {
                                        at(nz, q) = __fadd_rn(__fmul_rn(bz, at(oz, q)), __fmul_rn(az, Dz[q]));
                                        at(jz, q) = __fadd_rn(Dz[q], at(nz, q));
                                        at(vz, q) = __fsub_rn(at(vz, q), __fmul_rn(at(a2, q), at(jz, q)));
                                    }
                                }
                                stg4(A.psi_out + po + 2 * g.plane, nx);
                                stg4(A.psi_out + po + 3 * g.plane, nz);
                            } else if (need) {
                                const float4 k2 = ldg4(A.k2 + o);
                                const float4 k3 = ldg4(A.k3 + o);
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    const int gx = gx0 + q;
                                    if (vx_row && gx >= g.vx_c0 && gx <= g.vx_c1) {
                                        at(vx, q) = __fmaf_rn(-at(a2, q), Dx[q], (1.f - at(k2, q)) * at(vx, q));
                                        at(jx, q) = Dx[q];
                                    }
                                    if (vz_row && gx >= g.vz_c0 && gx <= g.vz_c1) {
                                        at(vz, q) = __fmaf_rn(-at(a2, q), Dz[q], (1.f - at(k3, q)) * at(vz, q));
                                        at(jz, q) = Dz[q];
                                    }
                                }
                            }
                        }
                        if (IMG == 2 && imaging) {
                            store_img4(imaging, (long long)s * g.plane + A.img_field_stride + o, A.img_fmt, jx);
                            store_img4(imaging, (long long)s * g.plane + 2 * A.img_field_stride + o, A.img_fmt,
                                       jz);
                        }
                        float *outs = A.out + (long long)s * 3 * g.plane + o;
                        stg4(outs, pv);
                        stg4(outs + g.plane, vx);
                        stg4(outs + 2 * g.plane, vz);
                        if (has_rcv) {
                            sts4(sVX + rr * VXW + 4 * lane + 4, vx);
                            sts4(sVZ + (rv + 2 * R) * RW + 4 * lane, vz);
                        }
                        if (ENERGY && gz >= g.pml && gz < g.pml + g.nz) {
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const int gx = gx0 + q;
                                if (gx >= g.pml && gx < g.pml + g.nx) {
                                    at(e_p[u], q) = __fmaf_rn(at(pv, q), at(pv, q), at(e_p[u], q));
                                    at(e_vx[u], q) = __fmaf_rn(at(vx, q), at(vx, q), at(e_vx[u], q));
                                    at(e_vz[u], q) = __fmaf_rn(at(vz, q), at(vz, q), at(e_vz[u], q));
                                }
                            }
                        }
                    }
                }
            }
        }

        // ---------------- receivers of this tile ---------------------------
        if (has_rcv) {
            __syncthreads();
            for (int e = rcv0 + threadIdx.x; e < rcv1; e += NTHR) {
                const int4 en = A.rcv_ent[e];
                const int rr = en.x + R, cc = en.y + 4;
                const long long t = ((long long)s * g.nt + it) * g.n_rcv + en.z;
                if (en.w & 1) {
                    if (A.tr_p) A.tr_p[t] = sP[rr * RW + cc];
                    if (A.tr_vx) A.tr_vx[t] = sVX[rr * VXW + cc + 4];
                }
                if ((en.w & 2) && A.tr_vz) A.tr_vz[t] = sVZ[(en.x + 2 * R) * RW + cc];
            }
        }
        // order this iteration's generic-proxy shared-memory writes before the
        // TMA that refills the buffer (issued after the next iteration's
        // mid-shot barrier)
        fence_proxy_async_smem();
    }

    if (ENERGY && vlane && A.energy) {
        // add this CTA's partial sums (over its shots) into the padded maps
#pragma unroll
        for (int u = 0; u < G::LV; ++u) {
            const int gz = z0 + vb + u;
            if (u < vcnt && gz >= g.pml && gz < g.pml + g.nz && gx0 < g.Nx) {
                const long long o = (long long)gz * g.pitch + gx0;
                red_add_v4(A.energy + o, e_p[u]);
                red_add_v4(A.energy + g.plane + o, e_vx[u]);
                red_add_v4(A.energy + 2 * g.plane + o, e_vz[u]);
            }
        }
    }
}

// Single-model launch: blockIdx covers shot groups [grp0, grp0 + grp_count)
// of every tile (one launch for all groups, or one per group when the groups
// run on their own streams), in the order of the work list when there is one.
template <int R, int TZ, bool FS, bool ENERGY, int IMG>
__global__ void __launch_bounds__(NTHR, TZ <= 16 ? 2 : 1)
fwd_step_kernel(const __grid_constant__ CUtensorMap mP, const __grid_constant__ CUtensorMap mVX,
                const __grid_constant__ CUtensorMap mVZ, const __grid_constant__ CUtensorMap mA1,
                const __grid_constant__ CUtensorMap mA2, const FwdArgs A)
{
    int tile, s0, ns;
    if (A.items) {
        const int4 w = A.items[blockIdx.x];
        tile = w.x;
        s0 = w.y;
        ns = w.z;
    } else {
        const int group = A.grp0 + (int)(blockIdx.x % A.grp_count);
        tile = (int)(blockIdx.x / A.grp_count);
        s0 = group * A.g.shots_per_cta;
        ns = min(A.g.n_shots - s0, A.g.shots_per_cta);
    }
    fwd_body<R, TZ, FS, ENERGY, IMG>(&mP, &mVX, &mVZ, &mA1, &mA2, A, tile, s0, ns);
}

template <int R, int TZ>
constexpr size_t fwd_smem_bytes()
{
    return StepSmem<R, TZ>::BYTES;
}

// Per tile: 1 if the tile's rectangles need no masks (tile_is_interior) and
// see no damping (k1 on the p rectangle, k2 / k3 on the tile all zero).
template <int R, int TZ>
__global__ void tile_fast_kernel(const StepGeom g, const float *__restrict__ k1, const float *__restrict__ k2,
                                 const float *__restrict__ k3, int *flags, int4 still)
{
    const int tile = blockIdx.x;
    const int z0 = (tile / g.tiles_x) * TZ, x0 = (tile % g.tiles_x) * TX;
    // still: rows [x, y] x cols [z, w] where the CPML profiles vanish (the whole grid without CPML)
    bool ok = tile_is_interior<R, TZ>(g, z0, x0) && z0 - R >= still.x && z0 + TZ + R - 1 <= still.y &&
              x0 - 4 >= still.z && x0 + TX + 3 <= still.w;
    bool damped = false;
    if (ok) {
        for (int i = threadIdx.x; i < (TZ + 2 * R) * RW; i += blockDim.x) {
            const int r = i / RW, c = i % RW;
            const long long o = (long long)(z0 - R + r) * g.pitch + (x0 - 4 + c);
            damped |= k1[o] != 0.f;
            if (r >= R && r < R + TZ && c >= 4 && c < 4 + TX) damped |= (k2[o] != 0.f) || (k3[o] != 0.f);
        }
    }
    damped = __syncthreads_or(damped);
    if (threadIdx.x == 0) flags[tile] = (ok && !damped) ? 1 : 0;
}

}  // namespace gb
