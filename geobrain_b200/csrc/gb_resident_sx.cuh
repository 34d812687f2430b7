// Resident forward with one exchange per step (4th order, no free surface).
//
// The two-exchange resident kernel (gb_resident.cuh) waits twice a step for
// its neighbours: for their v cells before the p update and for their p
// cells before the v update.  Through global memory each wait costs about
// one L2 round trip, which on a small grid is most of the step.  Here a tile
// updates p also on R rows above and below it and R columns to each side
// (p of the neighbours' edge cells, computed again from the same inputs with
// the same arithmetic, so the same numbers), and then v on its own cells
// from that p; only v crosses tiles, once a step, to all eight neighbours
// (the corner cells come from the diagonal ones).  The rect holds 2R halo
// rows and the usual 4 halo columns of p, vx and vz:
//
//   rect rows [z0 - 2R, z0 + TZ + 2R), columns [x0 - 4, x0 + 124)
//   p update on rows [z0 - R, z0 + TZ + R), columns [x0 - 1, x0 + 122)
//   v update on the tile; v sent on its first and last 2R rows and its
//   first and last 4-column lanes
//
// and needs v at rows z0 - 2R .. z0 + TZ + 2R - 1 (vz) and columns x0 - 3 ..
// x0 + 122 (vx): all inside the rect for R = 2.  The exchange words are
// double-buffered by step parity: a tile may start step n + 1 (and write its
// step n + 1 words) while a neighbour still reads its step n words, but not
// step n + 2, which needs that neighbour's step n + 1 words.
#pragma once

#include "gb_resident.cuh"

namespace gb {

constexpr int kSxDirs = 8;   // strips by direction: up, down, left, right, up-left, up-right, down-left, down-right

template <int NW, int TZ>
struct SxGeo {
    static constexpr int R = 2, H = 2 * R;
    static constexpr int NTH = NW * 32;
    static constexpr int ROWS = TZ + 2 * H;       // rect rows [z0 - H, z0 + TZ + H)
    static constexpr int FL = ROWS * RS;
    static constexpr int PROWS = TZ + 2 * R;      // p-update rows [z0 - R, z0 + TZ + R); coefficient planes
    static constexpr int CF = PROWS * RS;
    static constexpr int NPITEM = PROWS * 30;     // 4-cell p items on lanes 1..30
    static constexpr int NVITEM = TZ * 30;        // 4-cell v items
    static constexpr int BAND = H * 30;           // 4-cell groups of an up / down strip, per field
    static constexpr int GROUPS = BAND > TZ ? BAND : TZ;              // groups per strip and field (slot size)
    static constexpr int SLOT = kSxDirs * 2 * GROUPS * 4;             // (value, tag) words of one parity
    static constexpr int NRECV = 2 * (2 * BAND + 2 * TZ + 4 * H);     // halo groups received per step (both fields)
    static constexpr int LE = (TZ + NW - 1) / NW;
    static constexpr size_t SMEM = size_t(3 * FL + 6 * CF) * 4;
};

// Word offset of group `g` of field `f` (0 vx, 1 vz) in strip `d` of a slot.
template <int NW, int TZ>
__device__ __forceinline__ int sx_word(int d, int f, int g)
{
    using G = SxGeo<NW, TZ>;
    return ((d * 2 + f) * G::GROUPS + g) * 4;
}

// Send the new vx, vz of tile item (rect row r, lane l) to the strips that
// hold it: up (tile rows 0 .. H-1), down (rows TZ-H .. TZ-1), left (lane 1),
// right (lane 30) and the four corners.  `my` is this tile's slot of the
// step's parity.
template <int NW, int TZ>
__device__ __forceinline__ void sx_send(uint2 *my, int r, int l, float4 vx, float4 vz, unsigned int tag,
                                        const int (&nb)[kSxDirs])
{
    using G = SxGeo<NW, TZ>;
    constexpr int H = G::H;
    const bool top = r < 2 * H, bot = r >= TZ;   // rect rows [H, 2H) / [TZ, TZ + H)
    auto put = [&](int d, int g) {
        if (nb[d] < 0) return;
        ll_put4(my + sx_word<NW, TZ>(d, 0, g), vx, tag);
        ll_put4(my + sx_word<NW, TZ>(d, 1, g), vz, tag);
    };
    if (top) put(0, (r - H) * 30 + l - 1);
    if (bot) put(1, (r - TZ) * 30 + l - 1);
    if (l == 1) {
        put(2, r - H);
        if (top) put(4, r - H);
        if (bot) put(6, r - TZ);
    }
    if (l == 30) {
        put(3, r - H);
        if (top) put(5, r - H);
        if (bot) put(7, r - TZ);
    }
}

// Halo group h (of NRECV) this tile receives: the source words (null where
// there is no neighbour) in the neighbour's slot, and the destination in vx
// (field 0) or vz (field 1).  Per field: the upper tile's down strip into
// rect rows [0, H), the lower tile's up strip into rows [TZ + H, TZ + 2H),
// the left tile's right strip into lane 0 of the tile rows, the right
// tile's left strip into lane 31, and the corners' strips into lanes 0 / 31
// of rows [0, H) and [TZ + H, TZ + 2H).
template <int NW, int TZ>
__device__ __forceinline__ const uint2 *sx_halo(int h, float *sVX, float *sVZ, const uint2 *slots, int par,
                                                const int (&nb)[kSxDirs], float *&dst)
{
    using G = SxGeo<NW, TZ>;
    constexpr int H = G::H, BAND = G::BAND, SEG = 2 * BAND + 2 * TZ + 4 * H;
    const int f = h / SEG, k = h % SEG;
    float *F = f == 0 ? sVX : sVZ;
    int d, sd, j;   // neighbour direction, its strip, group
    if (k < BAND) {
        d = 0; sd = 1; j = k;
        dst = F + (j / 30) * RS + 4 * (1 + j % 30);
    } else if (k < 2 * BAND) {
        d = 1; sd = 0; j = k - BAND;
        dst = F + (TZ + H + j / 30) * RS + 4 * (1 + j % 30);
    } else if (k < 2 * BAND + TZ) {
        d = 2; sd = 3; j = k - 2 * BAND;
        dst = F + (H + j) * RS;
    } else if (k < 2 * BAND + 2 * TZ) {
        d = 3; sd = 2; j = k - 2 * BAND - TZ;
        dst = F + (H + j) * RS + 124;
    } else {
        const int c = k - 2 * BAND - 2 * TZ;
        j = c % H;
        d = 4 + c / H;          // 4 UL, 5 UR, 6 DL, 7 DR
        sd = 11 - d;            // their DR, DL, UR, UL strips
        const int row = d < 6 ? j : TZ + H + j;
        dst = F + row * RS + ((d & 1) ? 124 : 0);
    }
    if (nb[d] < 0) return nullptr;
    return slots + ((size_t)nb[d] * 2 + par) * G::SLOT + sx_word<NW, TZ>(sd, f, j);
}

// Receive this step's halo: each round reads every group of this thread
// not yet arrived, all reads in flight together, then checks them, so a
// thread waits about one L2 round trip per round rather than per group
// (bounded; a give-up, or another CTA's error, sets the status word).
// Uniform outcome.
template <int NW, int TZ>
__device__ __forceinline__ bool sx_receive(float *sVX, float *sVZ, const uint2 *slots, int par,
                                           const int (&nb)[kSxDirs], unsigned int tag, int *err)
{
    using G = SxGeo<NW, TZ>;
    constexpr int NK = (G::NRECV + G::NTH - 1) / G::NTH;
    const uint2 *w[NK];
    float *dst[NK];
    unsigned int pending = 0;
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        const int h = threadIdx.x + k * G::NTH;
        w[k] = h < G::NRECV ? sx_halo<NW, TZ>(h, sVX, sVZ, slots, par, nb, dst[k]) : nullptr;
        if (w[k]) pending |= 1u << k;
    }
    bool ok = true;
    for (uint32_t i = 0; pending; ++i) {
        uint4 a[NK], b[NK];
#pragma unroll
        for (int k = 0; k < NK; ++k)
            if ((pending >> k) & 1u) {
                a[k] = ld_relaxed_u4(w[k]);
                b[k] = ld_relaxed_u4(w[k] + 2);
            }
#pragma unroll
        for (int k = 0; k < NK; ++k)
            if (((pending >> k) & 1u) && a[k].y == tag && a[k].w == tag && b[k].y == tag && b[k].w == tag) {
                sts4(dst[k], make_float4(__uint_as_float(a[k].x), __uint_as_float(a[k].z), __uint_as_float(b[k].x),
                                         __uint_as_float(b[k].z)));
                pending &= ~(1u << k);
            }
        if (!pending) break;
        if (i >= kMaxPolls) {
            atomicExch(err, -4);
            ok = false;
            break;
        }
        if (i > 64) {
            if (*reinterpret_cast<volatile int *>(err) != 0) {
                ok = false;
                break;
            }
            __nanosleep(32);
        }
    }
    return __syncthreads_and(ok);
}

// Pressure update of one cell (rect row r, rect column c) outside lanes
// 1..30: the arithmetic of divergence4 and res_p_cells for that cell.
__device__ __forceinline__ void sx_p_cell(const ResArgs &A, const ResCtx &C, int r, int c, int it)
{
    constexpr int R = 2;
    const StepGeom &g = A.g;
    const float *vx = C.sVX + r * RS, *vz = C.sVZ + c;
    float d = 0.f;
#pragma unroll
    for (int k = 0; k < R; ++k)
        d = __fmaf_rn(g.c[k], ((vx[c + k] - vx[c - 1 - k]) + vz[(r + k) * RS]) - vz[(r - 1 - k) * RS], d);
    float p = C.sP[r * RS + c];
    const float a1 = C.cA1[(r - R) * RS + c];
    p = C.fast ? __fmaf_rn(-a1, d, p) : __fmaf_rn(-a1, d, C.cD1[(r - R) * RS + c] * p);
    if (C.z0 - R + r == C.sz && C.x0 - 4 + c == C.sx) p = __fadd_rn(p, __fmul_rn(g.dt, A.wavelet[(long long)C.s * g.nt + it]));
    C.sP[r * RS + c] = p;
}

template <int NW, int TZ>
__global__ void __launch_bounds__(NW * 32, 1) resident_sx_kernel(const ResArgs A)
{
    using G = SxGeo<NW, TZ>;
    constexpr int R = G::R, H = G::H;
    extern __shared__ __align__(128) float sm[];
    ResCtx C;
    C.sP = sm;
    C.sVX = sm + G::FL;
    C.sVZ = sm + 2 * G::FL;
    float *cf = sm + 3 * G::FL;   // coefficient planes on rect rows [R, R + PROWS)
    C.cA1 = cf;
    C.cD1 = cf + G::CF;
    C.cA2X = cf + 2 * G::CF;
    C.cD2 = cf + 3 * G::CF;
    C.cA2Z = cf + 4 * G::CF;
    C.cD3 = cf + 5 * G::CF;
    float *sP = C.sP, *sVX = C.sVX, *sVZ = C.sVZ;
    const StepGeom &g = A.g;
    const int tile = (int)(blockIdx.x % A.n_tiles);
    const int s = A.shot0 + (int)(blockIdx.x / A.n_tiles);
    const int ti = tile / A.tiles_x, tj = tile % A.tiles_x;
    const int z0 = ti * TZ, x0 = tj * TX;
    C.z0 = z0 - R;   // rect row r is global row C.z0 - R + r = z0 - H + r
    C.x0 = x0;
    C.s = s;
    C.sz = A.src_z[s];
    C.sx = A.src_x[s];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *st = A.state + (long long)s * 3 * g.plane;
    uint2 *slots = A.xbuf + (size_t)s * A.n_tiles * 2 * G::SLOT;
    const bool up = ti > 0, dn = ti + 1 < A.tiles_z, lf = tj > 0, rt = tj + 1 < A.tiles_x;
    const int nb[kSxDirs] = {up ? tile - A.tiles_x : -1,          dn ? tile + A.tiles_x : -1,
                             lf ? tile - 1 : -1,                  rt ? tile + 1 : -1,
                             up && lf ? tile - A.tiles_x - 1 : -1, up && rt ? tile - A.tiles_x + 1 : -1,
                             dn && lf ? tile + A.tiles_x - 1 : -1, dn && rt ? tile + A.tiles_x + 1 : -1};

    // the state's rect (zero off the grid)
    for (int e = threadIdx.x; e < G::ROWS * 32; e += G::NTH) {
        const int r = e >> 5, l = e & 31;
        const int gz = z0 - H + r, gx = x0 - 4 + 4 * l;
        const bool in = gz >= 0 && gz < g.Nz && gx >= 0 && gx < g.pitch;
        const long long o = (long long)gz * g.pitch + gx;
        sts4(sP + r * RS + 4 * l, in ? ld4(st + o) : zero4());
        sts4(sVX + r * RS + 4 * l, in ? ld4(st + g.plane + o) : zero4());
        sts4(sVZ + r * RS + 4 * l, in ? ld4(st + 2 * g.plane + o) : zero4());
    }
    // coefficients of the p-update rows, masks and damping folded in
    bool damped = false;
    for (int e = threadIdx.x; e < G::PROWS * 32; e += G::NTH) {
        const int pr = e >> 5, l = e & 31;
        const int gz = z0 - R + pr, gx0 = x0 - 4 + 4 * l;
        const bool in = gz >= 0 && gz < g.Nz && gx0 >= 0 && gx0 < g.pitch;
        const long long o = (long long)gz * g.pitch + gx0;
        const float4 a1 = in ? ldg4(A.a1 + o) : zero4(), a2 = in ? ldg4(A.a2 + o) : zero4();
        const float4 k1 = in ? ldg4(A.k1 + o) : zero4(), k2 = in ? ldg4(A.k2 + o) : zero4();
        const float4 k3 = in ? ldg4(A.k3 + o) : zero4();
        float4 a1m, d1, a2x, d2, a2z, d3;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int gx = gx0 + q;
            const bool pm = gz >= g.p_r0 && gz <= g.p_r1 && gx >= g.p_c0 && gx <= g.p_c1;
            const bool xm = gz >= g.vx_r0 && gz <= g.vx_r1 && gx >= g.vx_c0 && gx <= g.vx_c1;
            const bool zm = gz >= g.vz_r0 && gz <= g.vz_r1 && gx >= g.vz_c0 && gx <= g.vz_c1;
            at(a1m, q) = pm ? at(a1, q) : 0.f;
            at(d1, q) = pm ? 1.f - at(k1, q) : 1.f;
            at(a2x, q) = xm ? at(a2, q) : 0.f;
            at(d2, q) = xm ? 1.f - at(k2, q) : 1.f;
            at(a2z, q) = zm ? at(a2, q) : 0.f;
            at(d3, q) = zm ? 1.f - at(k3, q) : 1.f;
        }
        const int c = pr * RS + 4 * l;
        sts4(cf + c, a1m);
        sts4(cf + G::CF + c, d1);
        sts4(cf + 2 * G::CF + c, a2x);
        sts4(cf + 3 * G::CF + c, d2);
        sts4(cf + 4 * G::CF + c, a2z);
        sts4(cf + 5 * G::CF + c, d3);
        damped |= k1.x != 0.f || k1.y != 0.f || k1.z != 0.f || k1.w != 0.f || k2.x != 0.f || k2.y != 0.f ||
                  k2.z != 0.f || k2.w != 0.f || k3.x != 0.f || k3.y != 0.f || k3.z != 0.f || k3.w != 0.f;
    }
    // the undamped update where every cell this tile updates is inside the
    // masks and no cell it reads coefficients of is damped
    const bool inside = z0 - R >= g.p_r0 && z0 + TZ + R - 1 <= g.p_r1 && x0 - 1 >= g.p_c0 &&
                        x0 + TX + 1 <= g.p_c1 && z0 >= g.vx_r0 && z0 + TZ - 1 <= g.vx_r1 && x0 >= g.vx_c0 &&
                        x0 + TX - 1 <= g.vx_c1 && z0 >= g.vz_r0 && z0 + TZ - 1 <= g.vz_r1 && x0 >= g.vz_c0 &&
                        x0 + TX - 1 <= g.vz_c1;
    C.fast = !__syncthreads_or(damped) && inside;
    const int rcv0 = A.rcv_ptr[tile], rcv1 = A.rcv_ptr[tile + 1];
    const bool has_rcv = rcv1 > rcv0 && (A.tr_p || A.tr_vx || A.tr_vz);
    uint32_t emask = 0;
    if (A.energy && lane >= 1 && lane <= 30) {
        const int gx0 = x0 - 4 + 4 * lane;
#pragma unroll
        for (int u = 0; u < G::LE; ++u) {
            const int gz = z0 + warp + NW * u;
            if (warp + NW * u < TZ && gz >= g.pml && gz < g.pml + g.nz && gz < g.Nz && gx0 < g.Nx)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (gx0 + q >= g.pml && gx0 + q < g.pml + g.nx) emask |= 1u << (4 * u + q);
        }
    }
    float4 e_p[G::LE], e_vx[G::LE], e_vz[G::LE];
#pragma unroll
    for (int u = 0; u < G::LE; ++u) e_p[u] = e_vx[u] = e_vz[u] = zero4();
    __syncthreads();

    for (int it = A.it0; it < A.it1; ++it) {
        // ---- p on rows [z0 - R, z0 + TZ + R), columns [x0 - 1, x0 + 122) ----
        for (int i = threadIdx.x; i < G::NPITEM + 3 * G::PROWS; i += G::NTH) {
            if (i < G::NPITEM) {
                const int r = R + i / 30, l = 1 + i % 30;
                float4 wz[2 * R];
#pragma unroll
                for (int t = 0; t < 2 * R; ++t) wz[t] = lds4(sVZ + (r - R + t) * RS + 4 * l);
                res_p_cells<R>(A, C, r, l, wz, 0, it);
            } else {
                // the cells of the neighbours' edge lanes: column 3, 124 and 125
                const int j = i - G::NPITEM, r = R + j / 3, k = j % 3;
                sx_p_cell(A, C, r, k == 0 ? 3 : 123 + k, it);
            }
        }
        __syncthreads();
        // ---- v on the tile, sent on as computed -------------------------------
        const bool send = it + 1 < A.it1;
        uint2 *my = slots + ((size_t)tile * 2 + (it & 1)) * G::SLOT;
        for (int i = threadIdx.x; i < G::NVITEM; i += G::NTH) {
            const int r = H + i / 30, l = 1 + i % 30;
            float4 wp[2 * R];
#pragma unroll
            for (int t = 0; t < 2 * R; ++t) wp[t] = lds4(sP + (r - R + 1 + t) * RS + 4 * l);
            float4 vx, vz;
            res_v_cells<R>(A, C, r, l, wp, 0, vx, vz);
            if (send) sx_send<NW, TZ>(my, r, l, vx, vz, tag_v(it), nb);
        }
        __syncthreads();
        // ---- receivers of this tile (acoustic_2d.py:272-274), energy -------
        if (has_rcv) {
            for (int e = rcv0 + threadIdx.x; e < rcv1; e += G::NTH) {
                const int4 en = A.rcv_ent[e];
                const int o = (en.x + H) * RS + en.y + 4;
                const long long t = ((long long)s * g.nt + it) * g.n_rcv + en.z;
                if (A.tr_p) A.tr_p[t] = sP[o];
                if (A.tr_vx) A.tr_vx[t] = sVX[o];
                if (A.tr_vz) A.tr_vz[t] = sVZ[o];
            }
        }
        if (emask) {
#pragma unroll
            for (int u = 0; u < G::LE; ++u) {
                if (((emask >> (4 * u)) & 15u) == 0) continue;
                const int r = H + warp + NW * u;
                const float4 pv = lds4(sP + r * RS + 4 * lane), vx = lds4(sVX + r * RS + 4 * lane);
                const float4 vz = lds4(sVZ + r * RS + 4 * lane);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if ((emask >> (4 * u + q)) & 1u) {
                        at(e_p[u], q) = __fmaf_rn(at(pv, q), at(pv, q), at(e_p[u], q));
                        at(e_vx[u], q) = __fmaf_rn(at(vx, q), at(vx, q), at(e_vx[u], q));
                        at(e_vz[u], q) = __fmaf_rn(at(vz, q), at(vz, q), at(e_vz[u], q));
                    }
                }
            }
        }
        // ---- the neighbours' new v around the tile (the halo cells only) ----
        if (send) {
            if (!sx_receive<NW, TZ>(sVX, sVZ, slots, it & 1, nb, tag_v(it), A.err)) return;
        } else {
            __syncthreads();
        }
    }

    // the owned cells back to the state; the energy sums into the padded maps
    for (int e = threadIdx.x; e < TZ * 32; e += G::NTH) {
        const int r = e >> 5, l = e & 31;
        const int gz = z0 + r, gx = x0 - 4 + 4 * l;
        if (l >= 1 && l <= 30 && gz < g.Nz && gx < g.pitch) {
            const long long o = (long long)gz * g.pitch + gx;
            stg4(st + o, lds4(sP + (H + r) * RS + 4 * l));
            stg4(st + g.plane + o, lds4(sVX + (H + r) * RS + 4 * l));
            stg4(st + 2 * g.plane + o, lds4(sVZ + (H + r) * RS + 4 * l));
        }
    }
    if (A.energy && lane >= 1 && lane <= 30) {
        const int gx0 = x0 - 4 + 4 * lane;
#pragma unroll
        for (int u = 0; u < G::LE; ++u) {
            const int gz = z0 + warp + NW * u;
            if (warp + NW * u < TZ && gz >= g.pml && gz < g.pml + g.nz && gx0 < g.Nx) {
                const long long o = (long long)gz * g.pitch + gx0;
                red_add_v4(A.energy_map + o, e_p[u]);
                red_add_v4(A.energy_map + g.plane + o, e_vx[u]);
                red_add_v4(A.energy_map + 2 * g.plane + o, e_vz[u]);
            }
        }
    }
}

}  // namespace gb
