// Resident forward: a persistent kernel whose CTAs keep their tile of the
// wavefield, and the tile's coefficients, in shared memory for every time
// step of a launch.
//
// The tile kernel (gb_fwd.cuh) streams the whole state through HBM once per
// step, which is what a many-shot run needs.  With one shot, or a small
// grid, a step is a few microseconds of work spread over too few CTAs, and
// the per-step launch, the pipeline fill and the p-halo recompute dominate
// (the 100 x 200 forward runs at 3 % of the HBM roofline that way).  Here
// one launch runs many steps; each CTA owns a 120-column x TZ-row tile of
// one shot and holds p, vx, vz on the tile plus an R-cell halo, and six
// coefficient planes on the tile.
//
// The cells of a tile split into a boundary (the R rows at the top and at the
// bottom, and the 4-column strips at the left and right) and an interior.
// An interior cell's update reads only the tile's own cells; a boundary
// cell's reads the halo.  The neighbours (the four edge tiles: the stencils
// are axis-aligned) need only the boundary cells, and a boundary cell is
// sent to them by the thread that computes it, straight from its
// registers.  So a step runs
//
//   p interior;  receive the neighbours' v boundary cells of the previous
//   step into the halo;  p boundary (sending each cell on), source,
//   free-surface mirror;  v interior;  receive the p boundary cells;
//   v boundary (sending on), mirror;  receivers and energy,
//
// and the time a boundary cell takes to reach the neighbours is spent on
// interior work.  The cell arithmetic is the tile kernel's, tap for tap (the
// same stencil helpers and update expressions), so the traces are the same
// numbers bit for bit.
//
// Two ways to send:
//   * Global memory, flag in the data: every float goes out as an 8-byte
//     (value, tag) word, the tag naming the step and field, with relaxed
//     GPU-scope stores and no fence; the receiver polls its words until
//     every tag is the expected one.  One L2 trip from sender to receiver, no flag
//     round trip.  Every CTA must be resident at once (a cooperative
//     launch), and every poll is bounded: a receiver that gives up, or sees
//     another CTA's error, sets the status word and the launch ends.
//   * Distributed shared memory, when one shot's tiles fit in one
//     thread-block cluster (16 CTAs at most): the sender stores into the
//     neighbour's halo, and the two exchanges of a step are the two halves
//     of the hardware cluster barrier (arrive after the boundary cells,
//     wait before the neighbours' are read), with the interior work between
//     them.  No cooperative launch: each shot is one cluster, and clusters
//     never wait on each other.
//
// The damping and the update masks are folded into the coefficient planes
// at the start of a launch: a1m = a1 where p is updated, else 0; d1 = 1 - k1
// where p is updated, else 1; likewise a2x, d2 (vx) and a2z, d3 (vz).  A
// damped or masked cell then runs p' = fma(-a1m, D, d1 * p), the tile
// kernel's damped update where the mask holds, and p' = p (up to the sign
// of a zero) where it does not; tiles with no mask and no damping run the
// undamped update fma(-a1, D, p).
#pragma once

#include "gb_fwd.cuh"

namespace gb {

// Row stride of the resident rects: 128 columns and 4 floats of padding, so
// that the same column of consecutive rows falls in different shared-memory
// bank groups (the boundary items at lanes 1 and 30 run down a column).
constexpr int RS = 132;
constexpr int kResParts = 8;   // strips per tile: p top / bottom / left / right, vz top / bottom, vx left / right

template <int R, int NW, int TZ>
struct ResGeo {
    static constexpr int NTH = NW * 32;
    static constexpr int ROWS = TZ + 2 * R;       // rect rows [z0 - R, z0 + TZ + R)
    static constexpr int FL = ROWS * RS;          // floats of one field rect (128 wide: cols [x0 - 4, x0 + 124))
    static constexpr int CF = TZ * RS;            // floats of one coefficient plane on the owned rows
    static constexpr int NCOEF = 6;               // a1m, d1, a2x, d2, a2z, d3
    static constexpr int RP = R * 30;             // 4-cell groups of a row strip (R rows, lanes 1..30)
    static constexpr int CP = TZ;                 // 4-cell groups of a column strip
    static constexpr int PART = 4 * (RP > CP ? RP : CP);             // (value, tag) words per strip slot
    static constexpr int NHALO = 2 * RP + 2 * CP;                    // 4-cell halo groups received per exchange
    static constexpr int NI = TZ > 2 * R ? TZ - 2 * R : 0;           // interior rows: rect rows [2R, TZ)
    static constexpr int LI = (NI + NW - 1) / NW;                    // interior rows per warp
    static constexpr int NB = TZ - NI;                               // boundary rows (all lanes)
    static constexpr int NITEM = NB * 30 + NI * 2;                   // boundary items of 4 cells
    static constexpr int LE = (TZ + NW - 1) / NW;                    // energy rows per warp
    static constexpr size_t SMEM = size_t(3 * FL + NCOEF * CF) * 4;
};

struct ResArgs {
    StepGeom g;                       // grid, masks, taps, dt, nt, n_rcv, plane, pitch
    int tiles_x, tiles_z, n_tiles;    // the resident tiling (TX columns, TZ rows)
    int shot0;                        // first shot of this launch; blockIdx.x / n_tiles adds to it
    int it0, it1;                     // the time steps this launch runs
    int energy, free_surface;
    const float *a1, *k1, *a2, *k2, *k3;
    float *state;                     // [S][3][plane], read at the start and written at the end
    const int *src_z, *src_x;         // padded source cells
    const float *wavelet;             // [S][nt]
    const int *rcv_ptr;               // CSR over resident tiles
    const int4 *rcv_ent;              // (row in tile, col in tile, receiver, 0)
    float *tr_p, *tr_vx, *tr_vz;      // [S][nt][n_rcv] or null
    float *energy_map;                // [3][plane] padded accumulators (with energy)
    uint2 *xbuf;                      // [S][n_tiles][kResParts][PART] (value, tag) words, zero before a run
    int *err;
};

// Plain (coherent) 16-byte global load, for state another kernel wrote.
__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }

// Tags of the (value, tag) words: p boundary of step it, v boundary of step
// it (never 0, the value a run's strips start from).
__device__ __forceinline__ unsigned int tag_p(int it) { return 2u * (unsigned)it + 1u; }
__device__ __forceinline__ unsigned int tag_v(int it) { return 2u * (unsigned)it + 2u; }

// 4 cells as (value, tag) words: two 16-byte stores of two 8-byte words
// each; a reader sees each 8-byte word whole.  Relaxed at GPU scope: the
// words stay in L2 (system-scope volatile stores were written through to
// DRAM, 2.8 MB a step on the 400 x 1200 grid).
__device__ __forceinline__ void ll_put4(uint2 *w, float4 v, unsigned int tag)
{
    asm volatile("st.relaxed.gpu.global.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(w), "r"(__float_as_uint(v.x)), "r"(tag),
                 "r"(__float_as_uint(v.y)), "r"(tag)
                 : "memory");
    asm volatile("st.relaxed.gpu.global.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(w + 2), "r"(__float_as_uint(v.z)),
                 "r"(tag), "r"(__float_as_uint(v.w)), "r"(tag)
                 : "memory");
}

__device__ __forceinline__ void ll_put1(uint2 *w, float v, unsigned int tag)
{
    asm volatile("st.relaxed.gpu.global.v2.u32 [%0], {%1, %2};" ::"l"(w), "r"(__float_as_uint(v)), "r"(tag) : "memory");
}

__device__ __forceinline__ uint4 ld_relaxed_u4(const uint2 *w)
{
    uint4 r;
    asm volatile("ld.relaxed.gpu.global.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "l"(w)
                 : "memory");
    return r;
}

// Polls 4 cells' words until all four tags are `tag` (bounded).  A give-up,
// or another CTA's error seen while polling, sets the status word and
// returns false.
__device__ __forceinline__ bool ll_get4(const uint2 *w, unsigned int tag, float4 &v, int *err)
{
    for (uint32_t i = 0;; ++i) {
        const uint4 a = ld_relaxed_u4(w), b = ld_relaxed_u4(w + 2);
        if (a.y == tag && a.w == tag && b.y == tag && b.w == tag) {
            v = make_float4(__uint_as_float(a.x), __uint_as_float(a.z), __uint_as_float(b.x), __uint_as_float(b.z));
            return true;
        }
        if (i >= kMaxPolls) {
            atomicExch(err, -4);
            return false;
        }
        if (i > 64) {
            if (*reinterpret_cast<volatile int *>(err) != 0) return false;
            __nanosleep(32);
        }
    }
}

// Cluster barrier halves (every thread of every CTA of the cluster takes
// part; the hardware barrier needs no bound: every CTA runs the same
// sequence of arrivals and waits, which a launch of whole clusters keeps
// co-scheduled).
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

// The shared-memory address of local location `p` in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_map(const float *p, int rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}

__device__ __forceinline__ void st_cluster4(uint32_t addr, float4 v)
{
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(v.x), "f"(v.y), "f"(v.z),
                 "f"(v.w)
                 : "memory");
}

__device__ __forceinline__ void st_cluster1(uint32_t addr, float v)
{
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}

// What the cell updates of one CTA share.  Coefficient planes (owned rows,
// 128-wide rows like the fields): cA1 a1m, cD1 d1, cA2X a2x, cD2 d2,
// cA2Z a2z, cD3 d3.
struct ResCtx {
    float *sP, *sVX, *sVZ;
    const float *cA1, *cD1, *cA2X, *cD2, *cA2Z, *cD3;
    int z0, x0, s, sz, sx;
    bool fast;
};

// Pressure update of the 4 cells of rect row r, lane l (acoustic_2d.py
// :211-237), as the tile kernel computes it; wz[u + R] is vz row r.
// Returns the new values (also stored).
template <int R>
__device__ __forceinline__ float4 res_p_cells(const ResArgs &A, const ResCtx &C, int r, int l, const float4 *wz, int u,
                                              int it)
{
    const StepGeom &g = A.g;
    float4 pv = lds4(C.sP + r * RS + 4 * l);
    const float4 a1 = lds4(C.cA1 + (r - R) * RS + 4 * l);
    float D[4];
    divergence4<R>(C.sVX + r * RS - 4, l, wz, u, g.c, D);
    if (C.fast) {
#pragma unroll
        for (int q = 0; q < 4; ++q) at(pv, q) = __fmaf_rn(-at(a1, q), D[q], at(pv, q));
    } else {
        const float4 d1 = lds4(C.cD1 + (r - R) * RS + 4 * l);
#pragma unroll
        for (int q = 0; q < 4; ++q) at(pv, q) = __fmaf_rn(-at(a1, q), D[q], at(d1, q) * at(pv, q));
    }
    const int gx0 = C.x0 - 4 + 4 * l;
    if (C.z0 - R + r == C.sz && C.sx >= gx0 && C.sx < gx0 + 4) {
        // p + dt * w, rounded after the product and after the sum (acoustic_2d.py:230-233)
        const float amp = __fmul_rn(g.dt, A.wavelet[(long long)C.s * g.nt + it]);
        const int q = C.sx - gx0;
        if (q == 0) pv.x = __fadd_rn(pv.x, amp);
        else if (q == 1) pv.y = __fadd_rn(pv.y, amp);
        else if (q == 2) pv.z = __fadd_rn(pv.z, amp);
        else pv.w = __fadd_rn(pv.w, amp);
    }
    sts4(C.sP + r * RS + 4 * l, pv);
    return pv;
}

// Velocity update of the 4 cells of rect row r, lane l (acoustic_2d.py
// :244-265), as the tile kernel computes it; wp[u + R] is p row r + 1.
// Returns the new vx and vz (also stored).
template <int R>
__device__ __forceinline__ void res_v_cells(const ResArgs &A, const ResCtx &C, int r, int l, const float4 *wp, int u,
                                            float4 &vx, float4 &vz)
{
    const StepGeom &g = A.g;
    float Dx[4], Dz[4];
    float4 pv;
    grad_x4<R>(C.sP + r * RS, l, g.c, Dx, pv);
    grad_z4<R>(wp, u, g.c, Dz);
    vx = lds4(C.sVX + r * RS + 4 * l);
    vz = lds4(C.sVZ + r * RS + 4 * l);
    const int o = (r - R) * RS + 4 * l;
    const float4 ax = lds4(C.cA2X + o);
    if (C.fast) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            at(vx, q) = __fmaf_rn(-at(ax, q), Dx[q], at(vx, q));
            at(vz, q) = __fmaf_rn(-at(ax, q), Dz[q], at(vz, q));
        }
    } else {
        const float4 d2 = lds4(C.cD2 + o), az = lds4(C.cA2Z + o), d3 = lds4(C.cD3 + o);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            at(vx, q) = __fmaf_rn(-at(ax, q), Dx[q], at(d2, q) * at(vx, q));
            at(vz, q) = __fmaf_rn(-at(az, q), Dz[q], at(d3, q) * at(vz, q));
        }
    }
    sts4(C.sVX + r * RS + 4 * l, vx);
    sts4(C.sVZ + r * RS + 4 * l, vz);
}

// Boundary item i -> (rect row, lane): the boundary rows with lanes 1..30,
// then the interior rows with lanes 1 and 30.
template <int R, int NW, int TZ>
__device__ __forceinline__ void res_item(int i, int &r, int &l)
{
    using G = ResGeo<R, NW, TZ>;
    if (i < G::NB * 30) {
        const int b = i / 30;
        l = 1 + i % 30;
        r = (G::NI == 0 || b < R) ? R + b : TZ + (b - R);
    } else {
        const int j = i - G::NB * 30;
        r = 2 * R + (j >> 1);
        l = (j & 1) ? 30 : 1;
    }
}

// Where a CTA's boundary cells go: its neighbours (up, down, left, right;
// -1 for none), the neighbours' shared-memory field rects (cluster mode), or
// its own strips of (value, tag) words (global mode).
struct ResLinks {
    int nb[4];
    uint32_t rP[4], rVX[4], rVZ[4];   // neighbours' sP / sVX / sVZ in the cluster window
    uint2 *my;                        // this tile's kResParts strips
    int part;                         // words per strip
};

// Rect row r of this tile as the neighbours see it: row r + TZ of the upper
// tile (r in [R, 2R)), row r - TZ of the lower tile (r in [TZ, TZ + R));
// lane 1 of this tile is lane 31 of the left tile, lane 30 is lane 0 of the
// right tile.  Strip word offsets: rows (r - R) * 30 + l - 1 (top strip) or
// (r - TZ) * 30 + l - 1 (bottom strip), columns r - R; 4 words per group.

// Send the 4 cells (r, l) of field rect `f` (strips pr, pr + 1 for the rows
// and pc, pc + 1 for the columns; rows / cols false skips either).
template <int R, int TZ, bool CL>
__device__ __forceinline__ void res_send4(const ResLinks &K, const uint32_t (&rf)[4], int pr, int pc, bool rows,
                                          bool cols, int r, int l, float4 v, unsigned int tag)
{
    if (rows && r < 2 * R && K.nb[0] >= 0) {
        if (CL) st_cluster4(rf[0] + 4u * ((r + TZ) * RS + 4 * l), v);
        else ll_put4(K.my + pr * K.part + 4 * ((r - R) * 30 + l - 1), v, tag);
    }
    if (rows && r >= TZ && K.nb[1] >= 0) {
        if (CL) st_cluster4(rf[1] + 4u * ((r - TZ) * RS + 4 * l), v);
        else ll_put4(K.my + (pr + 1) * K.part + 4 * ((r - TZ) * 30 + l - 1), v, tag);
    }
    if (cols && l == 1 && K.nb[2] >= 0) {
        if (CL) st_cluster4(rf[2] + 4u * (r * RS + 124), v);
        else ll_put4(K.my + pc * K.part + 4 * (r - R), v, tag);
    }
    if (cols && l == 30 && K.nb[3] >= 0) {
        if (CL) st_cluster4(rf[3] + 4u * (r * RS), v);
        else ll_put4(K.my + (pc + 1) * K.part + 4 * (r - R), v, tag);
    }
}

// One cell (rect row r, column c = 4 l + q) of a mirror row, sent the same way.
template <int R, int TZ, bool CL>
__device__ __forceinline__ void res_send1(const ResLinks &K, const uint32_t (&rf)[4], int pr, int pc, bool cols, int r,
                                          int c, float v, unsigned int tag)
{
    const int l = c >> 2, q = c & 3;
    if (l < 1 || l > 30) return;
    if (r < 2 * R && K.nb[0] >= 0) {
        if (CL) st_cluster1(rf[0] + 4u * ((r + TZ) * RS + c), v);
        else ll_put1(K.my + pr * K.part + 4 * ((r - R) * 30 + l - 1) + q, v, tag);
    }
    if (r >= TZ && K.nb[1] >= 0) {
        if (CL) st_cluster1(rf[1] + 4u * ((r - TZ) * RS + c), v);
        else ll_put1(K.my + (pr + 1) * K.part + 4 * ((r - TZ) * 30 + l - 1) + q, v, tag);
    }
    if (cols && l == 1 && K.nb[2] >= 0) {
        if (CL) st_cluster1(rf[2] + 4u * (r * RS + 124 + q), v);
        else ll_put1(K.my + pc * K.part + 4 * (r - R) + q, v, tag);
    }
    if (cols && l == 30 && K.nb[3] >= 0) {
        if (CL) st_cluster1(rf[3] + 4u * (r * RS + q), v);
        else ll_put1(K.my + (pc + 1) * K.part + 4 * (r - R) + q, v, tag);
    }
}

// Global mode: the halo groups a thread receives, h = threadIdx.x + k NTH:
// rows of `rows_f` from the upper tile's bottom strip and the lower tile's
// top strip, columns 0..3 / 124..127 of `cols_f` from the left tile's right
// strip and the right tile's left strip (strips pb .. pb + 3 of each tile).
// Returns the source words, or null where there is no neighbour.
template <int R, int NW, int TZ>
__device__ __forceinline__ const uint2 *res_halo(int h, float *rows_f, float *cols_f, const uint2 *xb,
                                                 const int (&nb)[4], int pb, float *&dst)
{
    using G = ResGeo<R, NW, TZ>;
    int t, part, j;
    if (h < G::RP) {
        t = nb[0]; part = pb + 1; j = h;
        dst = rows_f + (h / 30) * RS + 4 * (1 + h % 30);
    } else if (h < 2 * G::RP) {
        j = h - G::RP; t = nb[1]; part = pb;
        dst = rows_f + (TZ + R + j / 30) * RS + 4 * (1 + j % 30);
    } else if (h < 2 * G::RP + G::CP) {
        j = h - 2 * G::RP; t = nb[2]; part = pb + 3;
        dst = cols_f + (R + j) * RS;
    } else {
        j = h - 2 * G::RP - G::CP; t = nb[3]; part = pb + 2;
        dst = cols_f + (R + j) * RS + 124;
    }
    return t < 0 ? nullptr : xb + ((size_t)t * kResParts + part) * G::PART + 4 * j;
}

// Receives the neighbours' boundary cells of one field pair into the halo,
// polling each group's words for `tag`.  Uniform outcome.
template <int R, int NW, int TZ>
__device__ __forceinline__ bool res_receive(float *rows_f, float *cols_f, const uint2 *xb, const int (&nb)[4], int pb,
                                            unsigned int tag, int *err)
{
    using G = ResGeo<R, NW, TZ>;
    bool ok = true;
    for (int h = threadIdx.x; h < G::NHALO && ok; h += G::NTH) {
        float *dst;
        const uint2 *w = res_halo<R, NW, TZ>(h, rows_f, cols_f, xb, nb, pb, dst);
        if (!w) continue;
        float4 v;
        ok = ll_get4(w, tag, v, err);
        if (ok) sts4(dst, v);
    }
    return __syncthreads_and(ok);
}

// CL: exchange through distributed shared memory within one cluster per
// shot (the launch's cluster is the shot's n_tiles CTAs, rank = tile).
template <int R, int NW, int TZ, bool CL>
__global__ void __launch_bounds__(NW * 32, 1) resident_fwd_kernel(const ResArgs A)
{
    using G = ResGeo<R, NW, TZ>;
    extern __shared__ __align__(128) float sm[];
    ResCtx C;
    C.sP = sm;
    C.sVX = sm + G::FL;
    C.sVZ = sm + 2 * G::FL;
    float *cf = sm + 3 * G::FL;
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
    C.z0 = z0;
    C.x0 = x0;
    C.s = s;
    C.sz = A.src_z[s];
    C.sx = A.src_x[s];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *st = A.state + (long long)s * 3 * g.plane;
    const uint2 *xb = A.xbuf + (size_t)s * A.n_tiles * kResParts * G::PART;
    ResLinks K;
    K.nb[0] = ti > 0 ? tile - A.tiles_x : -1;
    K.nb[1] = ti + 1 < A.tiles_z ? tile + A.tiles_x : -1;
    K.nb[2] = tj > 0 ? tile - 1 : -1;
    K.nb[3] = tj + 1 < A.tiles_x ? tile + 1 : -1;
    K.my = A.xbuf + ((size_t)s * A.n_tiles + tile) * kResParts * G::PART;
    K.part = G::PART;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        K.rP[k] = K.rVX[k] = K.rVZ[k] = 0;
        if (CL && K.nb[k] >= 0) {
            K.rP[k] = cluster_map(sP, K.nb[k]);
            K.rVX[k] = cluster_map(sVX, K.nb[k]);
            K.rVZ[k] = cluster_map(sVZ, K.nb[k]);
        }
    }

    // the state's rect (zero off the grid)
    for (int e = threadIdx.x; e < G::ROWS * 32; e += G::NTH) {
        const int r = e >> 5, l = e & 31;
        const int gz = z0 - R + r, gx = x0 - 4 + 4 * l;
        const bool in = gz >= 0 && gz < g.Nz && gx >= 0 && gx < g.pitch;
        const long long o = (long long)gz * g.pitch + gx;
        sts4(sP + r * RS + 4 * l, in ? ld4(st + o) : zero4());
        sts4(sVX + r * RS + 4 * l, in ? ld4(st + g.plane + o) : zero4());
        sts4(sVZ + r * RS + 4 * l, in ? ld4(st + 2 * g.plane + o) : zero4());
    }
    // the coefficients of the owned rows with the update masks and the
    // damping folded in
    bool damped = false;
    for (int e = threadIdx.x; e < TZ * 32; e += G::NTH) {
        const int r = e >> 5, l = e & 31;
        const int gz = z0 + r, gx0 = x0 - 4 + 4 * l;
        const bool in = gz < g.Nz && gx0 >= 0 && gx0 < g.pitch;
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
        const int c = r * RS + 4 * l;
        sts4(cf + c, a1m);
        sts4(cf + G::CF + c, d1);
        sts4(cf + 2 * G::CF + c, a2x);
        sts4(cf + 3 * G::CF + c, d2);
        sts4(cf + 4 * G::CF + c, a2z);
        sts4(cf + 5 * G::CF + c, d3);
        if (l >= 1 && l <= 30)
            damped |= k1.x != 0.f || k1.y != 0.f || k1.z != 0.f || k1.w != 0.f || k2.x != 0.f || k2.y != 0.f ||
                      k2.z != 0.f || k2.w != 0.f || k3.x != 0.f || k3.y != 0.f || k3.z != 0.f || k3.w != 0.f;
    }
    // no masks anywhere on the owned cells, and no damping: the undamped update
    const bool inside = z0 >= g.p_r0 && z0 + TZ - 1 <= g.p_r1 && x0 >= g.p_c0 && x0 + TX - 1 <= g.p_c1 &&
                        z0 >= g.vx_r0 && z0 + TZ - 1 <= g.vx_r1 && x0 >= g.vx_c0 && x0 + TX - 1 <= g.vx_c1 &&
                        z0 >= g.vz_r0 && z0 + TZ - 1 <= g.vz_r1 && x0 >= g.vz_c0 && x0 + TX - 1 <= g.vz_c1;
    C.fast = !__syncthreads_or(damped) && inside;
    const int fs = g.fs;
    // free surface: rect row of the mirror row (the tiling keeps rows fs-1 .. fs+1 in one tile)
    const int rm = fs - 1 - (z0 - R);
    const bool fs_own = A.free_surface && fs - 1 >= z0 && fs - 1 < z0 + TZ;
    if (A.free_surface && rm >= 0 && rm + 1 < G::ROWS) {
        // the state may come without the vz mirror row (the tile kernel never stores it)
        for (int c = threadIdx.x; c < RW; c += G::NTH) sVZ[rm * RS + c] = sVZ[(rm + 1) * RS + c];
    }
    const int rcv0 = A.rcv_ptr[tile], rcv1 = A.rcv_ptr[tile + 1];
    const bool has_rcv = rcv1 > rcv0 && (A.tr_p || A.tr_vx || A.tr_vz);
    const bool ilane = lane >= 2 && lane <= 29;           // interior lanes
    const int ri = 2 * R + warp * G::LI;                  // first interior row of this warp
    const bool interior = G::NI > 0 && ilane && ri < TZ;  // this thread updates interior cells
    // energy: bit 4u + q set where cell q of this lane's energy row u is summed
    uint32_t emask = 0;
    if (A.energy && lane >= 1 && lane <= 30) {
        const int gx0 = x0 - 4 + 4 * lane;
#pragma unroll
        for (int u = 0; u < G::LE; ++u) {
            const int r = R + warp + NW * u;
            const int gz = z0 - R + r;
            if (r < R + TZ && gz >= g.pml && gz < g.pml + g.nz && gz < g.Nz && gx0 < g.Nx)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (gx0 + q >= g.pml && gx0 + q < g.pml + g.nx) emask |= 1u << (4 * u + q);
        }
    }
    float4 e_p[G::LE], e_vx[G::LE], e_vz[G::LE];
#pragma unroll
    for (int u = 0; u < G::LE; ++u) e_p[u] = e_vx[u] = e_vz[u] = zero4();
    __syncthreads();
    if (CL) cluster_arrive();   // the first step's v exchange waits on this phase

    for (int it = A.it0; it < A.it1; ++it) {
        // ---- p interior (reads the tile's own v only) ---------------------
        if (interior) {
            float4 wz[G::LI + 2 * R - 1];
#pragma unroll
            for (int t = 0; t < G::LI + 2 * R - 1; ++t) wz[t] = lds4(sVZ + (ri - R + t) * RS + 4 * lane);
#pragma unroll
            for (int u = 0; u < G::LI; ++u)
                if (ri + u < TZ) res_p_cells<R>(A, C, ri + u, lane, wz, u, it);
        }
        // ---- the neighbours' v boundary cells of the previous step ---------
        // (a mirror row arrives mirrored: its owner sends it after the mirror)
        if (CL) cluster_wait();
        else if (it > A.it0 && !res_receive<R, NW, TZ>(sVZ, sVX, xb, K.nb, 4, tag_v(it - 1), A.err)) return;
        // ---- p boundary (sent on as computed), mirror ----------------------
        for (int i = threadIdx.x; i < G::NITEM; i += G::NTH) {
            int r, l;
            res_item<R, NW, TZ>(i, r, l);
            float4 wz[2 * R];
#pragma unroll
            for (int t = 0; t < 2 * R; ++t) wz[t] = lds4(sVZ + (r - R + t) * RS + 4 * l);
            const float4 pv = res_p_cells<R>(A, C, r, l, wz, 0, it);
            if (!(fs_own && r == rm)) res_send4<R, TZ, CL>(K, K.rP, 0, 2, true, true, r, l, pv, tag_p(it));
        }
        __syncthreads();
        if (fs_own) {
            // p[fs-1] = -p[fs+1]  (acoustic_2d.py:240-241), on the owned
            // columns: the x-halo cells of row fs-1 are the neighbours' to set
            for (int c = 4 + threadIdx.x; c < 4 + TX; c += G::NTH) {
                const float v = -sP[(rm + 2) * RS + c];
                sP[rm * RS + c] = v;
                res_send1<R, TZ, CL>(K, K.rP, 0, 2, true, rm, c, v, tag_p(it));
            }
            __syncthreads();
        }
        if (CL) cluster_arrive();
        // ---- v interior (reads the tile's own p only) ---------------------
        if (interior) {
            float4 wp[G::LI + 2 * R - 1];
#pragma unroll
            for (int t = 0; t < G::LI + 2 * R - 1; ++t) wp[t] = lds4(sP + (ri - R + 1 + t) * RS + 4 * lane);
#pragma unroll
            for (int u = 0; u < G::LI; ++u)
                if (ri + u < TZ) {
                    float4 vx, vz;
                    res_v_cells<R>(A, C, ri + u, lane, wp, u, vx, vz);
                }
        }
        // ---- the neighbours' p boundary cells ------------------------------
        if (CL) cluster_wait();
        else if (!res_receive<R, NW, TZ>(sP, sP, xb, K.nb, 0, tag_p(it), A.err)) return;
        // ---- v boundary (sent on unless this is the launch's last step), mirror
        const bool send_v = it + 1 < A.it1;
        for (int i = threadIdx.x; i < G::NITEM; i += G::NTH) {
            int r, l;
            res_item<R, NW, TZ>(i, r, l);
            float4 wp[2 * R];
#pragma unroll
            for (int t = 0; t < 2 * R; ++t) wp[t] = lds4(sP + (r - R + 1 + t) * RS + 4 * l);
            float4 vx, vz;
            res_v_cells<R>(A, C, r, l, wp, 0, vx, vz);
            if (send_v) {
                res_send4<R, TZ, CL>(K, K.rVZ, 4, 6, !(fs_own && r == rm), false, r, l, vz, tag_v(it));
                res_send4<R, TZ, CL>(K, K.rVX, 4, 6, false, true, r, l, vx, tag_v(it));
            }
        }
        __syncthreads();
        if (fs_own) {
            // vz[fs-1] = vz[fs]  (acoustic_2d.py:268-269)
            for (int c = 4 + threadIdx.x; c < 4 + TX; c += G::NTH) {
                const float v = sVZ[(rm + 1) * RS + c];
                sVZ[rm * RS + c] = v;
                if (send_v) res_send1<R, TZ, CL>(K, K.rVZ, 4, 6, false, rm, c, v, tag_v(it));
            }
            __syncthreads();
        }
        // ---- receivers of this tile (acoustic_2d.py:272-274), energy -------
        if (has_rcv) {
            for (int e = rcv0 + threadIdx.x; e < rcv1; e += G::NTH) {
                const int4 en = A.rcv_ent[e];
                const int o = (en.x + R) * RS + en.y + 4;
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
                const int r = R + warp + NW * u;
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
        // the next step writes p, which the receivers and the energy sums read
        __syncthreads();
        if (CL) cluster_arrive();
    }
    // the neighbours may still be sending into this CTA's halo: none leaves
    // the cluster before all are done
    if (CL) cluster_wait();

    // the owned cells back to the state; the energy sums into the padded maps
    __syncthreads();
    for (int e = threadIdx.x; e < TZ * 32; e += G::NTH) {
        const int r = e >> 5, l = e & 31;
        const int gz = z0 + r, gx = x0 - 4 + 4 * l;
        if (l >= 1 && l <= 30 && gz < g.Nz && gx < g.pitch) {
            const long long o = (long long)gz * g.pitch + gx;
            stg4(st + o, lds4(sP + (R + r) * RS + 4 * l));
            stg4(st + g.plane + o, lds4(sVX + (R + r) * RS + 4 * l));
            stg4(st + 2 * g.plane + o, lds4(sVZ + (R + r) * RS + 4 * l));
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
