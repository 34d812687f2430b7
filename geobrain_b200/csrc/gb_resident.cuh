// Resident forward: a persistent kernel whose CTAs keep their tile of the
// wavefield, and the tile's coefficients, in shared memory for every time
// step of a launch.
//
// The tile kernel (gb_fwd.cuh) streams the whole state through HBM once per
// step, which is what a many-shot run needs.  With one shot, or a small
// grid, a step is a few microseconds of work spread over too few CTAs, and
// the per-step launch, the pipeline fill and the p-halo recompute dominate
// (the 100 x 200 forward runs at 3 % of the HBM roofline that way).  Here
// one cooperative launch runs many steps; each CTA owns a 120-column x TZ-row
// tile of one shot and holds p, vx, vz on the tile plus an R-cell halo, and
// a1, k1, a2, k2, k3 on the tile.
//
// The cells of a tile split into a boundary (the R rows at the top and at the
// bottom, and the 4-column strips at the left and right) and an interior.
// An interior cell's update reads only the tile's own cells; a boundary
// cell's reads the halo.  The neighbours (the four edge tiles: the stencils
// are axis-aligned) need only the boundary strips.  So a step runs
//
//   p interior;  wait for the neighbours' v strips of the previous step,
//   copy them into the halo;  p boundary, source, free-surface mirror;
//   post the p strips and raise the p flag;  v interior;  wait for the
//   neighbours' p strips, copy them in;  v boundary, mirror;  receivers and
//   energy;  post the v strips and raise the v flag,
//
// and the time a flag takes to reach the neighbours is spent on interior
// work.  The cell arithmetic is the tile kernel's, tap for tap (the same
// stencil helpers and update expressions), so the traces are the same
// numbers bit for bit.
//
// Every CTA must be resident at once: the launch is cooperative (one CTA per
// SM at most), and every wait on a neighbour's flag is bounded; a wait that
// gives up, or sees another CTA's error, sets the status word and returns.
//
// When one shot's tiles fit in one thread-block cluster (16 CTAs at most),
// the cluster variant (CL) exchanges through distributed shared memory
// instead: a CTA reads its neighbours' boundary rows and columns straight
// from their shared memory, and the two exchanges of a step become the two
// halves of hardware cluster barriers (arrive after posting, wait before
// reading), with the interior work between them.  No global strips, no
// flags, and no cooperative launch: each shot is one cluster, and clusters
// never wait on each other.
#pragma once

#include "gb_fwd.cuh"

namespace gb {

constexpr int kResParts = 8;       // exchange strips per tile: p top / bottom / left / right, vz top / bottom, vx left / right
constexpr int kResFlagStride = 64; // words per tile in the flag array: [0] p posted, [32] v posted (separate 128-byte lines)

template <int R, int NW, int TZ>
struct ResGeo {
    static constexpr int NTH = NW * 32;
    static constexpr int ROWS = TZ + 2 * R;       // rect rows [z0 - R, z0 + TZ + R)
    static constexpr int FL = ROWS * RW;          // floats of one field rect (128 wide: cols [x0 - 4, x0 + 124))
    static constexpr int CF = TZ * RW;            // floats of one coefficient plane on the owned rows
    static constexpr int PART = R * RW > TZ * 4 ? R * RW : TZ * 4;   // floats per exchange strip
    static constexpr int NI = TZ > 2 * R ? TZ - 2 * R : 0;           // interior rows: rect rows [2R, TZ)
    static constexpr int LI = (NI + NW - 1) / NW;                    // interior rows per warp
    static constexpr int NB = TZ - NI;                               // boundary rows (all lanes)
    static constexpr int NITEM = NB * 30 + NI * 2;                   // boundary items of 4 cells
    static constexpr int LE = (TZ + NW - 1) / NW;                    // energy rows per warp
    static constexpr size_t SMEM = size_t(3 * FL + 5 * CF) * 4;
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
    float *xbuf;                      // [S][n_tiles][kResParts][PART] exchange strips
    unsigned int *flags;              // [S][n_tiles][kResFlagStride], zero before the first launch of a run
    int *err;
};

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(unsigned int *p, unsigned int v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Plain (coherent) 16-byte global load, for state another kernel wrote.
__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }

// Waits (bounded) until each existing neighbour's flag word `slot` reaches
// `target`.  Threads 0..3 poll one neighbour each; the vote makes the
// outcome uniform and orders every thread's later reads after the acquire.
// A give-up, or another CTA's error seen while polling, sets the status word
// and returns false.
__device__ __forceinline__ bool res_wait(const unsigned int *fl, const int (&nb)[4], int slot, unsigned int target,
                                         int *err)
{
    bool ok = true;
    if (threadIdx.x < 4) {
        const int n = nb[threadIdx.x];
        if (n >= 0) {
            const unsigned int *f = fl + (size_t)n * kResFlagStride + slot;
            ok = false;
            for (uint32_t i = 0; i < kMaxPolls; ++i) {
                if (ld_acquire_gpu(f) >= target) {
                    ok = true;
                    break;
                }
                if (i > 256) {
                    if (*reinterpret_cast<volatile int *>(err) != 0) break;
                    __nanosleep(32);
                }
            }
            if (!ok) atomicExch(err, -4);
        }
    }
    return __syncthreads_and(ok);
}

// Post the tile's strips of one field pair: rows [R, 2R) and [TZ, TZ + R) of
// `rows_f` into parts (pr, pr + 1), columns 4..7 and 120..123 of the owned
// rows of `cols_f` into parts (pc, pc + 1), then (after the CTA barrier)
// raise the flag with one release store, which publishes every thread's
// strip stores that the barrier ordered before it.
template <int R, int NW, int TZ>
__device__ __forceinline__ void res_post(const float *rows_f, const float *cols_f, float *my, int pr, int pc,
                                         unsigned int *flag, unsigned int value)
{
    using G = ResGeo<R, NW, TZ>;
    float *top = my + pr * G::PART, *bot = my + (pr + 1) * G::PART;
    for (int e = threadIdx.x; e < R * 32; e += G::NTH) {
        const int r = e >> 5, l = e & 31;
        stg4(top + 4 * e, lds4(rows_f + (R + r) * RW + 4 * l));
        stg4(bot + 4 * e, lds4(rows_f + (TZ + r) * RW + 4 * l));
    }
    float *lft = my + pc * G::PART, *rgt = my + (pc + 1) * G::PART;
    for (int r = threadIdx.x; r < TZ; r += G::NTH) {
        stg4(lft + 4 * r, lds4(cols_f + (R + r) * RW + 4));
        stg4(rgt + 4 * r, lds4(cols_f + (R + r) * RW + 120));
    }
    __syncthreads();
    if (threadIdx.x == 0) st_release_gpu(flag, value);
}

// Copy the neighbours' strips into the halo: rows [0, R) from the upper
// tile's bottom strip, rows [TZ + R, TZ + 2R) from the lower tile's top strip,
// columns 0..3 / 124..127 of the owned rows from the left tile's right strip
// and the right tile's left strip.  L2 loads (the strips change every step).
template <int R, int NW, int TZ>
__device__ __forceinline__ void res_fetch(float *rows_f, float *cols_f, const float *xb, const int (&nb)[4], int pr,
                                          int pc)
{
    using G = ResGeo<R, NW, TZ>;
    const size_t tile_fl = (size_t)kResParts * G::PART;
    for (int e = threadIdx.x; e < R * 32; e += G::NTH) {
        const int r = e >> 5, l = e & 31;
        if (nb[0] >= 0)
            sts4(rows_f + r * RW + 4 * l, __ldcg(reinterpret_cast<const float4 *>(xb + nb[0] * tile_fl +
                                                                                  (pr + 1) * G::PART) + e));
        if (nb[1] >= 0)
            sts4(rows_f + (TZ + R + r) * RW + 4 * l,
                 __ldcg(reinterpret_cast<const float4 *>(xb + nb[1] * tile_fl + pr * G::PART) + e));
    }
    for (int r = threadIdx.x; r < TZ; r += G::NTH) {
        if (nb[2] >= 0)
            sts4(cols_f + (R + r) * RW,
                 __ldcg(reinterpret_cast<const float4 *>(xb + nb[2] * tile_fl + (pc + 1) * G::PART) + r));
        if (nb[3] >= 0)
            sts4(cols_f + (R + r) * RW + 124,
                 __ldcg(reinterpret_cast<const float4 *>(xb + nb[3] * tile_fl + pc * G::PART) + r));
    }
}

// Cluster barrier halves (every thread of every CTA of the cluster takes
// part; the hardware barrier needs no bound: every CTA runs the same
// sequence of arrivals and waits, which a launch of whole clusters keeps
// co-scheduled).
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

// The address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ const float *cluster_map(const float *p, int rank)
{
    uint64_t r;
    asm volatile("mapa.u64 %0, %1, %2;" : "=l"(r) : "l"(reinterpret_cast<uint64_t>(p)), "r"(rank));
    return reinterpret_cast<const float *>(r);
}

// The neighbours' boundary rows and columns copied from their shared memory
// into the halo (the cluster variant of res_fetch): rows [0, R) from the
// upper tile's rows [TZ, TZ + R), rows [TZ + R, TZ + 2R) from the lower
// tile's rows [R, 2R), columns 0..3 / 124..127 from the left tile's columns
// 120..123 / the right tile's columns 4..7 (owned rows).
template <int R, int NW, int TZ>
__device__ __forceinline__ void res_fetch_cluster(float *rows_f, float *cols_f, const int (&nb)[4])
{
    using G = ResGeo<R, NW, TZ>;
    for (int e = threadIdx.x; e < R * 32; e += G::NTH) {
        const int r = e >> 5, l = e & 31;
        if (nb[0] >= 0) sts4(rows_f + r * RW + 4 * l, lds4(cluster_map(rows_f + (TZ + r) * RW + 4 * l, nb[0])));
        if (nb[1] >= 0)
            sts4(rows_f + (TZ + R + r) * RW + 4 * l, lds4(cluster_map(rows_f + (R + r) * RW + 4 * l, nb[1])));
    }
    for (int r = threadIdx.x; r < TZ; r += G::NTH) {
        if (nb[2] >= 0) sts4(cols_f + (R + r) * RW, lds4(cluster_map(cols_f + (R + r) * RW + 120, nb[2])));
        if (nb[3] >= 0) sts4(cols_f + (R + r) * RW + 124, lds4(cluster_map(cols_f + (R + r) * RW + 4, nb[3])));
    }
}

// What the cell updates of one CTA share.
struct ResCtx {
    float *sP, *sVX, *sVZ;
    const float *cA1, *cK1, *cA2, *cK2, *cK3;
    int z0, x0, s, sz, sx;
    bool fast;
};

// Pressure update of the 4 cells of rect row r, lane l (acoustic_2d.py
// :211-237), as the tile kernel computes it; wz[u + R] is vz row r.
template <int R>
__device__ __forceinline__ void res_p_cells(const ResArgs &A, const ResCtx &C, int r, int l, const float4 *wz, int u,
                                            int it)
{
    const StepGeom &g = A.g;
    const int gz = C.z0 - R + r, gx0 = C.x0 - 4 + 4 * l;
    float4 pv = lds4(C.sP + r * RW + 4 * l);
    const float4 a1 = lds4(C.cA1 + (r - R) * RW + 4 * l);
    float D[4];
    if (C.fast) {
        divergence4<R>(C.sVX + r * RW - 4, l, wz, u, g.c, D);
#pragma unroll
        for (int q = 0; q < 4; ++q) at(pv, q) = __fmaf_rn(-at(a1, q), D[q], at(pv, q));
    } else if (gz >= g.p_r0 && gz <= g.p_r1 && gx0 + 3 >= g.p_c0 && gx0 <= g.p_c1) {
        divergence4<R>(C.sVX + r * RW - 4, l, wz, u, g.c, D);
        const float4 k1 = lds4(C.cK1 + (r - R) * RW + 4 * l);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int gx = gx0 + q;
            if (gx >= g.p_c0 && gx <= g.p_c1) at(pv, q) = __fmaf_rn(-at(a1, q), D[q], (1.f - at(k1, q)) * at(pv, q));
        }
    }
    if (gz == C.sz && C.sx >= gx0 && C.sx < gx0 + 4) {
        // p + dt * w, rounded after the product and after the sum (acoustic_2d.py:230-233)
        const float amp = __fmul_rn(g.dt, A.wavelet[(long long)C.s * g.nt + it]);
        const int q = C.sx - gx0;
        if (q == 0) pv.x = __fadd_rn(pv.x, amp);
        else if (q == 1) pv.y = __fadd_rn(pv.y, amp);
        else if (q == 2) pv.z = __fadd_rn(pv.z, amp);
        else pv.w = __fadd_rn(pv.w, amp);
    }
    sts4(C.sP + r * RW + 4 * l, pv);
}

// Velocity update of the 4 cells of rect row r, lane l (acoustic_2d.py
// :244-265), as the tile kernel computes it; wp[u + R] is p row r + 1.
template <int R>
__device__ __forceinline__ void res_v_cells(const ResArgs &A, const ResCtx &C, int r, int l, const float4 *wp, int u)
{
    const StepGeom &g = A.g;
    const int gz = C.z0 - R + r, gx0 = C.x0 - 4 + 4 * l;
    if (!(C.fast || (gz < g.Nz && gx0 < g.Nx))) return;
    float Dx[4], Dz[4];
    float4 pv;
    grad_x4<R>(C.sP + r * RW, l, g.c, Dx, pv);
    grad_z4<R>(wp, u, g.c, Dz);
    float4 vx = lds4(C.sVX + r * RW + 4 * l);
    float4 vz = lds4(C.sVZ + r * RW + 4 * l);
    const float4 a2 = lds4(C.cA2 + (r - R) * RW + 4 * l);
    if (C.fast) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            at(vx, q) = __fmaf_rn(-at(a2, q), Dx[q], at(vx, q));
            at(vz, q) = __fmaf_rn(-at(a2, q), Dz[q], at(vz, q));
        }
    } else {
        const bool vx_row = gz >= g.vx_r0 && gz <= g.vx_r1;
        const bool vz_row = gz >= g.vz_r0 && gz <= g.vz_r1;
        if (!((vx_row && gx0 + 3 >= g.vx_c0 && gx0 <= g.vx_c1) || (vz_row && gx0 + 3 >= g.vz_c0 && gx0 <= g.vz_c1)))
            return;
        const float4 k2 = lds4(C.cK2 + (r - R) * RW + 4 * l);
        const float4 k3 = lds4(C.cK3 + (r - R) * RW + 4 * l);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int gx = gx0 + q;
            if (vx_row && gx >= g.vx_c0 && gx <= g.vx_c1)
                at(vx, q) = __fmaf_rn(-at(a2, q), Dx[q], (1.f - at(k2, q)) * at(vx, q));
            if (vz_row && gx >= g.vz_c0 && gx <= g.vz_c1)
                at(vz, q) = __fmaf_rn(-at(a2, q), Dz[q], (1.f - at(k3, q)) * at(vz, q));
        }
    }
    sts4(C.sVX + r * RW + 4 * l, vx);
    sts4(C.sVZ + r * RW + 4 * l, vz);
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
    float *cA1 = sm + 3 * G::FL;
    C.cA1 = cA1;
    C.cK1 = cA1 + G::CF;
    C.cA2 = cA1 + 2 * G::CF;
    C.cK2 = cA1 + 3 * G::CF;
    C.cK3 = cA1 + 4 * G::CF;
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
    float *xb = A.xbuf + (size_t)s * A.n_tiles * kResParts * G::PART;
    float *my = xb + (size_t)tile * kResParts * G::PART;
    unsigned int *fl = A.flags + (size_t)s * A.n_tiles * kResFlagStride;
    unsigned int *my_fl = fl + (size_t)tile * kResFlagStride;
    const int nb[4] = {ti > 0 ? tile - A.tiles_x : -1, ti + 1 < A.tiles_z ? tile + A.tiles_x : -1,
                       tj > 0 ? tile - 1 : -1, tj + 1 < A.tiles_x ? tile + 1 : -1};   // up, down, left, right

    // the state's rect (zero off the grid) and the coefficients of the owned rows
    for (int e = threadIdx.x; e < G::ROWS * 32; e += G::NTH) {
        const int r = e >> 5, l = e & 31;
        const int gz = z0 - R + r, gx = x0 - 4 + 4 * l;
        const bool in = gz >= 0 && gz < g.Nz && gx >= 0 && gx < g.pitch;
        const long long o = (long long)gz * g.pitch + gx;
        sts4(sP + r * RW + 4 * l, in ? ld4(st + o) : zero4());
        sts4(sVX + r * RW + 4 * l, in ? ld4(st + g.plane + o) : zero4());
        sts4(sVZ + r * RW + 4 * l, in ? ld4(st + 2 * g.plane + o) : zero4());
    }
    bool damped = false;
    for (int e = threadIdx.x; e < TZ * 32; e += G::NTH) {
        const int r = e >> 5, l = e & 31;
        const int gz = z0 + r, gx = x0 - 4 + 4 * l;
        const bool in = gz < g.Nz && gx >= 0 && gx < g.pitch;
        const long long o = (long long)gz * g.pitch + gx;
        const float4 k1 = in ? ldg4(A.k1 + o) : zero4(), k2 = in ? ldg4(A.k2 + o) : zero4();
        const float4 k3 = in ? ldg4(A.k3 + o) : zero4();
        sts4(cA1 + r * RW + 4 * l, in ? ldg4(A.a1 + o) : zero4());
        sts4(cA1 + 2 * G::CF + r * RW + 4 * l, in ? ldg4(A.a2 + o) : zero4());
        sts4(cA1 + G::CF + r * RW + 4 * l, k1);
        sts4(cA1 + 3 * G::CF + r * RW + 4 * l, k2);
        sts4(cA1 + 4 * G::CF + r * RW + 4 * l, k3);
        if (l >= 1 && l <= 30)
            damped |= k1.x != 0.f || k1.y != 0.f || k1.z != 0.f || k1.w != 0.f || k2.x != 0.f || k2.y != 0.f ||
                      k2.z != 0.f || k2.w != 0.f || k3.x != 0.f || k3.y != 0.f || k3.z != 0.f || k3.w != 0.f;
    }
    // no masks anywhere on the owned cells, and no damping: the branch-free path
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
        for (int c = threadIdx.x; c < RW; c += G::NTH) sVZ[rm * RW + c] = sVZ[(rm + 1) * RW + c];
    }
    const int rcv0 = A.rcv_ptr[tile], rcv1 = A.rcv_ptr[tile + 1];
    const bool has_rcv = rcv1 > rcv0 && (A.tr_p || A.tr_vx || A.tr_vz);
    const bool ilane = lane >= 2 && lane <= 29;           // interior lanes
    const int ri = 2 * R + warp * G::LI;                  // first interior row of this warp
    float4 e_p[G::LE], e_vx[G::LE], e_vz[G::LE];
#pragma unroll
    for (int u = 0; u < G::LE; ++u) e_p[u] = e_vx[u] = e_vz[u] = zero4();
    __syncthreads();
    if (CL) cluster_arrive();   // the first step's p exchange waits on this phase

    for (int it = A.it0; it < A.it1; ++it) {
        // ---- p interior (reads the tile's own v only) ---------------------
        if (G::NI > 0 && ilane && ri < TZ) {
            float4 wz[G::LI + 2 * R - 1];
#pragma unroll
            for (int t = 0; t < G::LI + 2 * R - 1; ++t) wz[t] = lds4(sVZ + (ri - R + t) * RW + 4 * lane);
#pragma unroll
            for (int u = 0; u < G::LI; ++u)
                if (ri + u < TZ) res_p_cells<R>(A, C, ri + u, lane, wz, u, it);
        }
        // ---- the neighbours' v strips of the previous step ----------------
        if (CL) {
            cluster_wait();
            if (it > A.it0) res_fetch_cluster<R, NW, TZ>(sVZ, sVX, nb);
        } else if (it > A.it0) {
            if (!res_wait(fl, nb, 32, (unsigned)it, A.err)) return;
            // (a mirror row in the halo arrives mirrored: its owner posts it after the mirror)
            res_fetch<R, NW, TZ>(sVZ, sVX, xb, nb, 4, 6);
        }
        __syncthreads();
        // ---- p boundary, free-surface mirror, post ------------------------
        for (int i = threadIdx.x; i < G::NITEM; i += G::NTH) {
            int r, l;
            res_item<R, NW, TZ>(i, r, l);
            float4 wz[2 * R];
#pragma unroll
            for (int t = 0; t < 2 * R; ++t) wz[t] = lds4(sVZ + (r - R + t) * RW + 4 * l);
            res_p_cells<R>(A, C, r, l, wz, 0, it);
        }
        __syncthreads();
        if (fs_own) {
            // p[fs-1] = -p[fs+1]  (acoustic_2d.py:240-241)
            for (int c = threadIdx.x; c < RW; c += G::NTH) sP[rm * RW + c] = -sP[(rm + 2) * RW + c];
            __syncthreads();
        }
        if (CL) cluster_arrive();
        else res_post<R, NW, TZ>(sP, sP, my, 0, 2, my_fl, (unsigned)it + 1u);
        // ---- v interior (reads the tile's own p only) ---------------------
        if (G::NI > 0 && ilane && ri < TZ) {
            float4 wp[G::LI + 2 * R - 1];
#pragma unroll
            for (int t = 0; t < G::LI + 2 * R - 1; ++t) wp[t] = lds4(sP + (ri - R + 1 + t) * RW + 4 * lane);
#pragma unroll
            for (int u = 0; u < G::LI; ++u)
                if (ri + u < TZ) res_v_cells<R>(A, C, ri + u, lane, wp, u);
        }
        // ---- the neighbours' p strips --------------------------------------
        if (CL) {
            cluster_wait();
            res_fetch_cluster<R, NW, TZ>(sP, sP, nb);
        } else {
            if (!res_wait(fl, nb, 0, (unsigned)it + 1u, A.err)) return;
            res_fetch<R, NW, TZ>(sP, sP, xb, nb, 0, 2);
        }
        __syncthreads();
        // ---- v boundary, mirror ---------------------------------------------
        for (int i = threadIdx.x; i < G::NITEM; i += G::NTH) {
            int r, l;
            res_item<R, NW, TZ>(i, r, l);
            float4 wp[2 * R];
#pragma unroll
            for (int t = 0; t < 2 * R; ++t) wp[t] = lds4(sP + (r - R + 1 + t) * RW + 4 * l);
            res_v_cells<R>(A, C, r, l, wp, 0);
        }
        __syncthreads();
        if (fs_own) {
            // vz[fs-1] = vz[fs]  (acoustic_2d.py:268-269)
            for (int c = threadIdx.x; c < RW; c += G::NTH) sVZ[rm * RW + c] = sVZ[(rm + 1) * RW + c];
            __syncthreads();
        }
        // ---- receivers of this tile (acoustic_2d.py:272-274), energy -------
        if (has_rcv) {
            for (int e = rcv0 + threadIdx.x; e < rcv1; e += G::NTH) {
                const int4 en = A.rcv_ent[e];
                const int o = (en.x + R) * RW + en.y + 4;
                const long long t = ((long long)s * g.nt + it) * g.n_rcv + en.z;
                if (A.tr_p) A.tr_p[t] = sP[o];
                if (A.tr_vx) A.tr_vx[t] = sVX[o];
                if (A.tr_vz) A.tr_vz[t] = sVZ[o];
            }
        }
        if (A.energy && lane >= 1 && lane <= 30) {
            const int gx0 = x0 - 4 + 4 * lane;
#pragma unroll
            for (int u = 0; u < G::LE; ++u) {
                const int r = R + warp + NW * u;
                const int gz = z0 - R + r;
                if (r < R + TZ && gz >= g.pml && gz < g.pml + g.nz && gz < g.Nz && gx0 < g.Nx) {
                    const float4 pv = lds4(sP + r * RW + 4 * lane), vx = lds4(sVX + r * RW + 4 * lane);
                    const float4 vz = lds4(sVZ + r * RW + 4 * lane);
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
        // ---- post the v strips ---------------------------------------------
        if (CL) cluster_arrive();
        else if (it + 1 < A.it1) res_post<R, NW, TZ>(sVZ, sVX, my, 4, 6, my_fl + 32, (unsigned)it + 1u);
    }
    // the neighbours may still be reading this CTA's rows: none leaves the
    // cluster before all are done
    if (CL) cluster_wait();

    // the owned cells back to the state; the energy sums into the padded maps
    __syncthreads();
    for (int e = threadIdx.x; e < TZ * 32; e += G::NTH) {
        const int r = e >> 5, l = e & 31;
        const int gz = z0 + r, gx = x0 - 4 + 4 * l;
        if (l >= 1 && l <= 30 && gz < g.Nz && gx < g.pitch) {
            const long long o = (long long)gz * g.pitch + gx;
            stg4(st + o, lds4(sP + (R + r) * RW + 4 * l));
            stg4(st + g.plane + o, lds4(sVX + (R + r) * RW + 4 * l));
            stg4(st + 2 * g.plane + o, lds4(sVZ + (R + r) * RW + 4 * l));
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
