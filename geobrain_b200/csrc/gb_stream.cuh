// Streaming forward step: the same update as fwd_step_kernel (gb_fwd.cuh),
// organised so that every pressure row is computed once per shot instead of
// once per tile plus a 2R-row halo.
//
// A CTA owns one column strip (120 columns, as the tiles) of one shot and a
// z-segment [zs, ze) of it, and walks down the segment in chunks of 16 rows.
// For chunk j (rows [a, a+16), a = zs + 16 j) it
//   1. updates p on the 16 rows [a+R, a+16+R): R rows ahead of the
//      velocities, so that
//   2. the v-stage of rows [a, a+16) finds every p row it needs, [a-R+1,
//      a+15+R], already updated: by this chunk or the one before.
// The state lives in shared-memory rings of three 16-row blocks per field:
//   p and vx blocks on the p grid  [zs - 16 + R + 16k, zs + R + 16k),
//   vz blocks on the v grid        [zs + 16k, zs + 16k + 16),
// and stage k = (p block k, vx block k, vz block k) arrives by TMA into slot
// k mod 3 while chunk k-2 computes.  A segment starts with a prologue that
// updates the p rows [zs-R, zs+R) (they belong to the segment above, which
// computes them too).  Free-surface models use the tile kernel.
//
// Per cell the arithmetic is the tile kernel's, operation for operation
// (the same stencil helpers and explicit roundings), so both give
// bit-identical fields.
#pragma once

#include "gb_fwd.cuh"

namespace gb {

constexpr int SCH = 16;                 // rows per chunk
constexpr int SRING = 3 * SCH;          // rows per ring
constexpr int SP_FL = SRING * RW;       // floats of the p ring
constexpr int SVX_FL = SRING * VXW;
constexpr int SVZ_FL = SRING * RW;
constexpr int SC_FL = 2 * SCH * RW;    // floats of an a1 or a2 ring (two blocks)
constexpr uint32_t kStageBytes = (uint32_t)(SCH * RW + SCH * VXW + SCH * RW + 2 * SCH * RW) * 4u;
constexpr uint32_t kVzBlockBytes = (uint32_t)(SCH * RW) * 4u;
constexpr size_t kStreamSmemBytes = (size_t)(SP_FL + SVX_FL + SVZ_FL + 2 * SC_FL) * 4 + 64;

struct StreamArgs {
    int shot0, n_shots;     // shots of this launch
    int n_seg, seg_chunks;  // z-segments per strip, chunks per segment
};

// slot of stage k (k >= -1) and the parity of its mbarrier phase: slot 2
// first serves the prologue's vz block -1
__device__ __forceinline__ int stage_slot(int k) { return (k + 3) % 3; }
__device__ __forceinline__ uint32_t stage_parity(int k)
{
    const int first = (k + 3) % 3 == 2 ? -1 : (k + 3) % 3;
    return (uint32_t)(((k - first) / 3) & 1);
}

__device__ __forceinline__ int ring_row(int z, int base)
{
    return (z - base) % SRING;   // z >= base for every row a segment touches
}

// Loads of stage k into its slot: p and vx block k (p grid), vz block k
// (v grid), and the coefficient blocks into two-block rings: a1 of p block k
// (slot k & 1) and a2 of v block k - 1 (slot (k - 1) & 1), so that the
// block a chunk uses is never the one being refilled.  `vz_only` for the
// prologue's vz block -1.
__device__ __forceinline__ void stream_stage_load(const CUtensorMap *mP, const CUtensorMap *mVX,
                                                  const CUtensorMap *mVZ, const CUtensorMap *mA1,
                                                  const CUtensorMap *mA2, float *sP, float *sVX, float *sVZ,
                                                  float *sA1, float *sA2, uint64_t *bars, int k, int zs, int x0,
                                                  int s, int R, bool vz_only)
{
    const int slot = stage_slot(k);
    uint64_t *bar = &bars[slot];
    mbar_arrive_expect_tx(bar, vz_only ? kVzBlockBytes : kStageBytes);
    if (!vz_only) {
        const int zp = zs - SCH + R + SCH * k;
        tma_load_3d(sP + slot * SCH * RW, mP, bar, x0 - 4, zp, 3 * s + 0);
        tma_load_3d(sVX + slot * SCH * VXW, mVX, bar, x0 - 8, zp, 3 * s + 1);
        tma_load_2d(sA1 + (k & 1) * SCH * RW, mA1, bar, x0 - 4, zp);
        tma_load_2d(sA2 + ((k + 1) & 1) * SCH * RW, mA2, bar, x0 - 4, zs + SCH * (k - 1));
    }
    tma_load_3d(sVZ + slot * SCH * RW, mVZ, bar, x0 - 4, zs + SCH * k, 3 * s + 2);
}

// p update of one warp's run of 2 rows starting at z (rows >= zlo and <
// zhi only), reading vz rows [z-R, z+1+R-1] from the vz ring.  The same
// arithmetic as fwd_body's p-stage.
template <int R, int IMG>
__device__ __forceinline__ void stream_p_rows(const FwdArgs &A, const StepGeom &g, int s, int it, int z, int zlo,
                                              int zhi, int zimg0, int zimg1, bool fast, float *sP, float *sVX,
                                              const float *sVZ, const float *sA1, int base_p, int base_vz, int lane,
                                              int gx0, bool vlane, int sz, int sx)
{
    float4 wz[2 + 2 * R - 1];
#pragma unroll
    for (int t = 0; t < 2 + 2 * R - 1; ++t) wz[t] = lds4(sVZ + ring_row(z - R + t, base_vz) * RW + 4 * lane);
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int gz = z + u;
        if (gz < zlo || gz >= zhi || gz < 0 || gz >= g.Nz) continue;
        const int pr = ring_row(gz, base_p);
        float4 pv = lds4(sP + pr * RW + 4 * lane);
        float D[4];
        const bool img_cell = IMG >= 1 && vlane && gz >= zimg0 && gz < zimg1;
        // a1 of this row: its p block k = (gz - base_p) / 16 sits in slot k & 1
        const float4 a1 = lds4(sA1 + ((((gz - base_p) >> 4) & 1) * SCH + ((gz - base_p) & (SCH - 1))) * RW + 4 * lane);
        if (fast) {
            divergence4<R>(sVX + pr * VXW, lane, wz, u, g.c, D);
#pragma unroll
            for (int q = 0; q < 4; ++q) at(pv, q) = __fmaf_rn(-at(a1, q), D[q], at(pv, q));
            if (img_cell && A.imaging)
                store_img4(A.imaging, (long long)s * g.plane + (long long)gz * g.pitch + gx0, A.img_fmt,
                           make_float4(-D[0], -D[1], -D[2], -D[3]));
        } else {
            const bool row_in = gz >= g.p_r0 && gz <= g.p_r1;
            if (row_in && (gx0 + 3 >= g.p_c0) && (gx0 <= g.p_c1)) {
                divergence4<R>(sVX + pr * VXW, lane, wz, u, g.c, D);
                const long long o = (long long)gz * g.pitch + gx0;
                const float4 k1 = ldg4(A.k1 + o);
                float4 img;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int gx = gx0 + q;
                    const bool m = gx >= g.p_c0 && gx <= g.p_c1;
                    at(img, q) = m ? -D[q] : 0.f;
                    if (m) at(pv, q) = __fmaf_rn(-at(a1, q), D[q], (1.f - at(k1, q)) * at(pv, q));
                }
                if (img_cell && A.imaging) store_img4(A.imaging, (long long)s * g.plane + o, A.img_fmt, img);
            }
        }
        if (gz == sz && sx >= gx0 && sx < gx0 + 4) {
            const float amp = __fmul_rn(g.dt, A.wavelet[(long long)s * g.nt + it]);
            const int q = sx - gx0;
            if (q == 0) pv.x = __fadd_rn(pv.x, amp);
            else if (q == 1) pv.y = __fadd_rn(pv.y, amp);
            else if (q == 2) pv.z = __fadd_rn(pv.z, amp);
            else pv.w = __fadd_rn(pv.w, amp);
        }
        sts4(sP + pr * RW + 4 * lane, pv);
    }
}

template <int R, bool ENERGY, int IMG>
__global__ void __launch_bounds__(NTHR, 2)
fwd_stream_kernel(const __grid_constant__ CUtensorMap mP, const __grid_constant__ CUtensorMap mVX,
                  const __grid_constant__ CUtensorMap mVZ, const __grid_constant__ CUtensorMap mA1,
                  const __grid_constant__ CUtensorMap mA2, const FwdArgs A, const StreamArgs SA)
{
    static_assert(2 * R <= SCH, "the prologue and the p-row lead need 2R <= 16");
    const StepGeom &g = A.g;
    extern __shared__ __align__(128) float smem[];
    float *sP = smem;
    float *sVX = sP + SP_FL;
    float *sVZ = sVX + SVX_FL;
    float *sA1 = sVZ + SVZ_FL;
    float *sA2 = sA1 + SC_FL;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sA2 + SC_FL);

    // work item: (strip, segment, shot)
    const int strip = (int)(blockIdx.x % g.tiles_x);
    const int seg = (int)((blockIdx.x / g.tiles_x) % SA.n_seg);
    const int s = SA.shot0 + (int)(blockIdx.x / ((unsigned)g.tiles_x * SA.n_seg));
    const int x0 = strip * TX;
    const int zs = seg * SA.seg_chunks * SCH;
    if (zs >= g.Nz) return;                                    // uniform per CTA
    const int n_chunks = min(SA.seg_chunks, (g.Nz - zs + SCH - 1) / SCH);
    const int ze = zs + n_chunks * SCH;                          // rows this CTA owns: [zs, min(ze, Nz))
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gx0 = x0 - 4 + 4 * lane;
    const bool vlane = lane >= 1 && lane <= 30;
    // ring row of a global row: block k of a field sits in slot (k + 3) % 3,
    // so the p / vx base is block 0's first row and the vz base lies three
    // blocks above block 0 (block -1 -> slot 2); every row touched is >= base
    const int base_p = zs - SCH + R, base_vz = zs - SRING;

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1);
        fence_mbar_init();
    }
    grid_dependency_wait();
    grid_launch_dependents();
    const int it = A.step_base ? *reinterpret_cast<const volatile int *>(A.step_base) + A.it : A.it;
    __syncthreads();
    if (threadIdx.x == 0) {
        stream_stage_load(&mP, &mVX, &mVZ, &mA1, &mA2, sP, sVX, sVZ, sA1, sA2, bars, -1, zs, x0, s, R, true);
        stream_stage_load(&mP, &mVX, &mVZ, &mA1, &mA2, sP, sVX, sVZ, sA1, sA2, bars, 0, zs, x0, s, R, false);
        stream_stage_load(&mP, &mVX, &mVZ, &mA1, &mA2, sP, sVX, sVZ, sA1, sA2, bars, 1, zs, x0, s, R, false);
    }
    const int sz = A.src_z[s], sx = A.src_x[s];
    const bool want_tr = A.tr_p || A.tr_vx || A.tr_vz;

    // ---- prologue: p rows [zs-R, zs+R) from stage 0 and vz block -1 -------
    {
        const bool ok = mbar_wait_bounded(&bars[2], 0) && mbar_wait_bounded(&bars[0], 0);
        if (!__syncthreads_and(ok)) {
            // give up uniformly, after waiting (bounded) for the three loads issued
            if (threadIdx.x == 0) {
                atomicExch(A.err, -4);
                for (int k = -1; k <= 1; ++k) mbar_wait_bounded(&bars[stage_slot(k)], stage_parity(k));
            }
            return;
        }
        if (warp < R)      // 2R rows, two per warp
            stream_p_rows<R, IMG>(A, g, s, it, zs - R + 2 * warp, zs - R, zs + R, zs, min(ze, g.Nz), false, sP,
                                  sVX, sVZ, sA1, base_p, base_vz, lane, gx0, vlane, sz, sx);
    }

    for (int j = 0; j < n_chunks; ++j) {
        const int a = zs + SCH * j;
        const int tile = (a / SCH) * g.tiles_x + strip;
        const bool fast = A.tile_fast[tile] != 0;
        // stage j+1 holds p / vx block j+1 and vz block j+1; the vote also
        // tells that every thread is done with chunk j-1 (slot of stage j+2)
        if (!__syncthreads_and(mbar_wait_bounded(&bars[stage_slot(j + 1)], stage_parity(j + 1)))) {
            // stage j+1 is the only load in flight here (j+2 is issued after this vote)
            if (threadIdx.x == 0) {
                atomicExch(A.err, -4);
                mbar_wait_bounded(&bars[stage_slot(j + 1)], stage_parity(j + 1));
            }
            return;
        }
        if (threadIdx.x == 0 && j + 2 <= n_chunks)
            stream_stage_load(&mP, &mVX, &mVZ, &mA1, &mA2, sP, sVX, sVZ, sA1, sA2, bars, j + 2, zs, x0, s, R, false);

        // ---- p-stage: rows [a+R, a+R+16) ------------------------------------
        stream_p_rows<R, IMG>(A, g, s, it, a + R + 2 * warp, a + R, a + R + SCH, zs, min(ze, g.Nz), fast, sP, sVX,
                              sVZ, sA1, base_p, base_vz, lane, gx0, vlane, sz, sx);
        __syncthreads();

        // ---- v-stage: rows [a, a+16), two per warp ---------------------------
        const int rcv0 = A.rcv_ptr[tile], rcv1 = A.rcv_ptr[tile + 1];
        const bool has_rcv = want_tr && rcv1 > rcv0;
        if (vlane) {
            const int z = a + 2 * warp;
            float4 wp[2 + 2 * R - 1];
#pragma unroll
            for (int t = 0; t < 2 + 2 * R - 1; ++t)
                wp[t] = lds4(sP + ring_row(z - R + 1 + t, base_p) * RW + 4 * lane);
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int gz = z + u;
                if (gz >= g.Nz || gz >= ze) continue;
                const int pr = ring_row(gz, base_p), vr = ring_row(gz, base_vz);
                float Dx[4], Dz[4];
                float4 pv;
                grad_x4<R>(sP + pr * RW, lane, g.c, Dx, pv);
                grad_z4<R>(wp, u, g.c, Dz);
                float4 vx = lds4(sVX + pr * VXW + 4 * lane + 4);
                float4 vz = lds4(sVZ + vr * RW + 4 * lane);
                const long long o = (long long)gz * g.pitch + gx0;
                float4 jx = zero4(), jz = zero4();
                const float4 a2 = lds4(sA2 + ((j & 1) * SCH + (gz - a)) * RW + 4 * lane);
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
                } else if (gx0 < g.Nx) {
                    const bool vx_row = gz >= g.vx_r0 && gz <= g.vx_r1;
                    const bool vz_row = gz >= g.vz_r0 && gz <= g.vz_r1;
                    const bool need = (vx_row && gx0 + 3 >= g.vx_c0 && gx0 <= g.vx_c1) ||
                                      (vz_row && gx0 + 3 >= g.vz_c0 && gx0 <= g.vz_c1);
                    if (need) {
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
                } else {
                    continue;
                }
                if (IMG == 2 && A.imaging) {
                    store_img4(A.imaging, (long long)s * g.plane + A.img_field_stride + o, A.img_fmt, jx);
                    store_img4(A.imaging, (long long)s * g.plane + 2 * A.img_field_stride + o, A.img_fmt, jz);
                }
                float *outs = A.out + (long long)s * 3 * g.plane + o;
                stg4(outs, pv);
                stg4(outs + g.plane, vx);
                stg4(outs + 2 * g.plane, vz);
                if (has_rcv) {
                    // vx / vz rows of this chunk are not read again: keep the new values for the receivers
                    sts4(sVX + pr * VXW + 4 * lane + 4, vx);
                    sts4(sVZ + vr * RW + 4 * lane, vz);
                }
                if (ENERGY && A.energy && gz >= g.pml && gz < g.pml + g.nz) {
                    float4 ep = zero4(), ex = zero4(), ez = zero4();
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int gx = gx0 + q;
                        if (gx >= g.pml && gx < g.pml + g.nx) {
                            at(ep, q) = __fmul_rn(at(pv, q), at(pv, q));
                            at(ex, q) = __fmul_rn(at(vx, q), at(vx, q));
                            at(ez, q) = __fmul_rn(at(vz, q), at(vz, q));
                        }
                    }
                    red_add_v4(A.energy + o, ep);
                    red_add_v4(A.energy + g.plane + o, ex);
                    red_add_v4(A.energy + 2 * g.plane + o, ez);
                }
            }
        }

        // ---- receivers of this chunk's tile ---------------------------------
        if (has_rcv) {
            __syncthreads();
            for (int e = rcv0 + threadIdx.x; e < rcv1; e += NTHR) {
                const int4 en = A.rcv_ent[e];
                const int zr = a + en.x, cc = en.y + 4;
                const long long t = ((long long)s * g.nt + it) * g.n_rcv + en.z;
                if (en.w & 1) {
                    if (A.tr_p) A.tr_p[t] = sP[ring_row(zr, base_p) * RW + cc];
                    if (A.tr_vx) A.tr_vx[t] = sVX[ring_row(zr, base_p) * VXW + cc + 4];
                }
                if ((en.w & 2) && A.tr_vz) A.tr_vz[t] = sVZ[ring_row(zr, base_vz) * RW + cc];
            }
        }
        // order this chunk's generic-proxy shared-memory writes before the TMA
        // that refills a slot (issued after the next chunk's vote)
        fence_proxy_async_smem();
    }
}

}  // namespace gb
