// Fused 3-D step: the pressure update, the source, both free-surface mirrors
// and the three velocity updates of one time step in ONE launch, with the
// reference's arithmetic (acoustic_3d.py:117-258, restated in gb_3d.cuh)
// rounded in the same order, so its state, traces, energies and imaging
// fields equal those of p3_kernel + v3_kernel bit for bit.
//
// A CTA owns TY rows (y) x 120 columns (x) of one shot and marches over the
// planes [zs, ze) of a z-chunk, reading the state before the step (`in`) and
// writing the state after it (`out`, a second buffer: neighbouring CTAs
// march at their own pace, so the update cannot run in place).
//
// Per plane zp (iteration j, zp = zs - 1 + j) one TMA stage brings, for the
// CTA's p rows y0-1 .. y0+TY+1 (the velocity updates' y halo) and 128
// columns x0-4 .. x0+123 (lanes 0 and 31 are the x halo):
//   p, vx of plane zp;  vz of plane zp+1;  a1, k1 of plane zp;
//   vy of plane zp on rows y0-3 .. y0+TY+2 (its y halo).
// Two stages alternate; the load of plane zp+2 is issued as soon as plane
// zp's stage is consumed.  Each thread keeps vz of planes zp-2 .. zp+1 of
// its 4 cells in registers (the z taps of the divergence); vx's x taps come
// from the neighbouring lanes by shuffles, vy's y taps from the stage.
//
// The new pressure of plane zp goes to a ring of 4 planes in shared memory.
// Two planes behind, the velocity phase updates plane zv = zp - 2 of the
// tile (warps 1..TY, lanes 1..30): its x and y taps read ring plane zv, its
// z taps ring planes zv-1 .. zv+2.  That phase writes all four fields of
// plane zv, so every cell of `out` the tile owns is written once.
//
// Energy maps (sum over shots of the squares, acoustic_3d.py:246-258): the
// shots of one tile form a thread-block cluster.  Each CTA leaves the
// squares of its plane in shared memory; after a cluster barrier, CTA r adds
// its share of the cells over the cluster's CTAs in shot order (distributed
// shared memory) and updates the maps with plain loads and stores, one owner
// per cell: the same sums, in the same order, as the per-thread shot loop of
// the split kernels.
#pragma once

#include "gb_3d.cuh"
#include "gb_device.cuh"

namespace gb {

constexpr int kF3MaxCluster = 8;   // shots per cluster (portable cluster size)

template <int TY>
struct F3Geo {
    static constexpr int PR = TY + 3;      // p rows: y0-1 .. y0+TY+1
    static constexpr int YR = TY + 6;      // vy rows: y0-3 .. y0+TY+2
    static constexpr int NT = PR * 32;     // one warp per p row
    // registers per thread: 8-row tiles run 2 CTAs (22 warps) per SM, at most
    // 6 warps per SM sub-partition of 16K registers; 16-row tiles 1 CTA of 19
    static constexpr int MAXREG = TY <= 8 ? 80 : 96;
    static constexpr int ROW = 128;        // floats per staged row
    static constexpr int S_P = 0;
    static constexpr int S_VX = PR * ROW;
    static constexpr int S_VZ = 2 * PR * ROW;
    static constexpr int S_A1 = 3 * PR * ROW;
    static constexpr int S_K1 = 4 * PR * ROW;
    static constexpr int S_VY = 5 * PR * ROW;
    static constexpr int STAGE_FL = 5 * PR * ROW + YR * ROW;
    static constexpr uint32_t STAGE_BYTES = STAGE_FL * 4u;
    static constexpr int RING_FL = 4 * PR * ROW;          // new p of 4 planes
    static constexpr int E_FL = 4 * TY * 32 * 4;          // squares [field][tile row][lane] float4
    static constexpr int E_ITEMS = 4 * TY * 30;           // (field, row, lane 1..30) per plane
    static constexpr size_t SMEM = (size_t)(2 * STAGE_FL + RING_FL + E_FL) * 4 + 16;
    static_assert((PR * ROW * 4) % 128 == 0 && (YR * ROW * 4) % 128 == 0, "TMA destinations 128-byte aligned");
};

struct Fused3Args {
    Geo3 g;
    int it;
    int shot0, ns;                   // shots [shot0, shot0 + ns) in this launch, fastest in blockIdx.x
    int tiles_x, tiles_y, chunk;     // tiles and z-chunk length (planes)
    int free_surface;
    const float *in;                 // [S][4][vol] state before the step
    float *out;                      // state after the step
    const float *a2, *k2, *k3, *k4;  // coefficient volumes
    const int *src;                  // [3][S] padded z, y, x
    const float *wavelet;            // [S][nt]
    float *energy[4];                // (nz, ny, nx) maps, or null (then no cluster is used)
    float *img_i, *img_j;            // imaging fields of this step (gradient), or null
    int *err;
};

// 4-D tiled TMA load (x, y, z, field plane); x a multiple of 4, the others
// may lie outside the map (zero fill).
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z,
                                            int w)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
        : "memory");
}

// Cluster barrier halves.  The warps that wrote squares arrive with release
// semantics (their shared-memory writes must reach the other CTAs); the
// others arrive relaxed, so they do not wait for their global stores.
__device__ __forceinline__ void f3_cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void f3_cluster_arrive_relaxed()
{
    asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void f3_cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

__device__ __forceinline__ float4 f3_ld_cluster4(const float *local, int rank)
{
    uint32_t a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(local)), "r"(rank));
    float4 v;
    asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"(a)
                 : "memory");
    return v;
}

__device__ __forceinline__ float4 sq4(const float4 &v)
{
    return make_float4(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y), __fmul_rn(v.z, v.z), __fmul_rn(v.w, v.w));
}

// Adds plane zr's squares over the cluster's CTAs, in shot order, into the
// energy maps: CTA `rank` of the cluster takes every ns-th (field, tile row,
// lane) item, spread over the 96 threads of its three halo warps (hid).  No
// barrier inside: the caller brackets it.
template <int TY>
__device__ __forceinline__ void f3_energy_reduce(const Fused3Args &A, const float *ebuf, int rank, int zr, int y0,
                                                 int x0, int hid)
{
    using G = F3Geo<TY>;
    const Geo3 &g = A.g;
    if (zr < g.pml || zr >= g.pml + g.nz) return;
    for (int it = rank + A.ns * hid; it < G::E_ITEMS; it += A.ns * 96) {
        const int f = it / (TY * 30), rest = it - f * (TY * 30);
        const int row = rest / 30, lane = 1 + rest % 30;
        const int y = y0 + row;
        if (y < g.pml || y >= g.pml + g.ny) continue;
        const float *e = ebuf + ((f * TY + row) * 32 + lane) * 4;
        float4 sum = f3_ld_cluster4(e, 0);
        for (int r = 1; r < A.ns; ++r) {
            const float4 v = f3_ld_cluster4(e, r);
            sum = make_float4(__fadd_rn(sum.x, v.x), __fadd_rn(sum.y, v.y), __fadd_rn(sum.z, v.z),
                              __fadd_rn(sum.w, v.w));
        }
        float *map = A.energy[f] + ((long long)(zr - g.pml) * g.ny + (y - g.pml)) * g.nx - g.pml;
        const int gx0 = x0 - 4 + 4 * lane;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int x = gx0 + q;
            if (x >= g.pml && x < g.pml + g.nx) map[x] = __fadd_rn(map[x], at(sum, q));
        }
    }
}

// IMG: 0 none; 1 I = -(dvx + dvy + dvz) on the p mask; 2 also dp/dx, dp/dy,
// dp/dz on the velocity masks (the density gradient).  Grid: one CTA per
// (z-chunk, tile row, tile column, shot), shot fastest; with ENERGY the
// launch's ns shots of a tile form one cluster.
template <int TY, bool ENERGY, int IMG>
__global__ void __maxnreg__(F3Geo<TY>::MAXREG)
step3_fused_kernel(const __grid_constant__ CUtensorMap mS,   // `in`: [4S][Nz][Ny][pitch], box 128 x PR
                   const __grid_constant__ CUtensorMap mY,   // `in`, box 128 x YR
                   const __grid_constant__ CUtensorMap mC,   // coefficients [6][Nz][Ny][pitch], box 128 x PR
                   const Fused3Args A)
{
    using G = F3Geo<TY>;
    constexpr int PRF = G::PR * G::ROW;    // one ring plane
    constexpr unsigned FULL = 0xffffffffu;
    const Geo3 &g = A.g;
    extern __shared__ __align__(128) float sm[];
    float *ring = sm + 2 * G::STAGE_FL;
    float *ebuf = ring + G::RING_FL;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ebuf + G::E_FL);

    int b = blockIdx.x;
    const int rank = b % A.ns;
    b /= A.ns;
    const int tx = b % A.tiles_x;
    b /= A.tiles_x;
    const int ty = b % A.tiles_y;
    const int zs = (b / A.tiles_y) * A.chunk;
    const int ze = min(g.Nz, zs + A.chunk);
    const int s = A.shot0 + rank;
    const int x0 = tx * TX, y0 = ty * TY;
    const int lane = threadIdx.x & 31, pr = threadIdx.x >> 5;
    const int y = y0 - 1 + pr;
    const int gx0 = x0 - 4 + 4 * lane;
    const bool vwarp = pr >= 1 && pr <= TY;
    const int hid = (pr == 0 ? 0 : pr - TY) * 32 + lane;   // halo warps 0, TY+1, TY+2: 0 .. 95
    const bool own = vwarp && lane >= 1 && lane <= 30 && y < g.Ny && gx0 < g.Nx;
    const bool cell_ok = y >= 0 && y < g.Ny && gx0 >= 0 && gx0 < g.pitch;
    const long long rowo = (long long)y * g.pitch + gx0;   // dereferenced for in-grid cells only
    const float *inS = A.in + (long long)s * 4 * g.vol;
    float *outS = A.out + (long long)s * 4 * g.vol;
    const int n_it = ze - zs + 3;                          // p planes zs-1 .. ze+1
    const bool fs_on = A.free_surface != 0 && g.fs >= 1;
    const int so = pr * G::ROW + 4 * lane;

    auto issue = [&](int zp, int k) {
        float *st = sm + k * G::STAGE_FL;
        mbar_arrive_expect_tx(&bars[k], G::STAGE_BYTES);
        tma_load_4d(st + G::S_P, &mS, &bars[k], x0 - 4, y0 - 1, zp, 4 * s + 0);
        tma_load_4d(st + G::S_VX, &mS, &bars[k], x0 - 4, y0 - 1, zp, 4 * s + 1);
        tma_load_4d(st + G::S_VZ, &mS, &bars[k], x0 - 4, y0 - 1, zp + 1, 4 * s + 3);
        tma_load_4d(st + G::S_A1, &mC, &bars[k], x0 - 4, y0 - 1, zp, 0);
        tma_load_4d(st + G::S_K1, &mC, &bars[k], x0 - 4, y0 - 1, zp, 1);
        tma_load_4d(st + G::S_VY, &mY, &bars[k], x0 - 4, y0 - 3, zp, 4 * s + 2);
    };
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        issue(zs - 1, 0);
        issue(zs, 1);
    }
    // vz of planes zs-3 .. zs-1 at this thread's cells (the z taps of the first p plane)
    float4 vzq[4];
    vzq[0] = zero4();
#pragma unroll
    for (int k = 1; k < 4; ++k) {
        const int z = zs - 4 + k;
        vzq[k] = (cell_ok && z >= 0 && z < g.Nz) ? ldg4(inS + 3 * g.vol + (long long)z * g.plane + rowo) : zero4();
    }
    const int sz = A.src[s], sy = A.src[g.n_shots + s], sx = A.src[2 * g.n_shots + s];
    const bool src_here = sy == y && sx >= gx0 && sx < gx0 + 4;
    const float amp = __fmul_rn(g.dt, A.wavelet[(long long)s * g.nt + A.it]);
    if (ENERGY) f3_cluster_arrive_relaxed();

    bool live = true;   // false once a stage wait gave up (the results are then void)
    for (int j = 0; j < n_it; ++j) {
        const int zp = zs - 1 + j, zv = zp - 2;
        const int k = j & 1;
        // the velocity phase's global loads of plane zv, issued before the
        // stage wait and the pressure phase that hide their latency
        float4 vx = zero4(), vy = zero4(), a2 = zero4(), k2 = zero4(), k3 = zero4(), k4 = zero4();
        if (own && j >= 3) {
            const long long o = (long long)zv * g.plane + rowo;
            vx = ldg4(inS + g.vol + o);
            vy = ldg4(inS + 2 * g.vol + o);
            a2 = ldg4(A.a2 + o);
            k2 = ldg4(A.k2 + o);
            k3 = ldg4(A.k3 + o);
            k4 = ldg4(A.k4 + o);
        }
        if (live && !mbar_wait_bounded(&bars[k], (j >> 1) & 1)) {
            live = false;
            atomicExch(A.err, -4);
        }
        const float *st = sm + k * G::STAGE_FL;

        // ---- pressure of plane zp on all p rows (tile + y / x halo) --------
        vzq[0] = vzq[1];
        vzq[1] = vzq[2];
        vzq[2] = vzq[3];
        vzq[3] = lds4(st + G::S_VZ + so);
        float4 p = lds4(st + G::S_P + so);
        {
            const float4 xc = lds4(st + G::S_VX + so);
            const float xl2 = __shfl_up_sync(FULL, xc.z, 1);
            const float xl1 = __shfl_up_sync(FULL, xc.w, 1);
            const float xr = __shfl_down_sync(FULL, xc.x, 1);
            if (zp >= g.fs + 1 && zp < g.Nz - 2 && y >= 2 && y < g.Ny - 2) {
                const float xs[7] = {xl2, xl1, xc.x, xc.y, xc.z, xc.w, xr};   // xs[q + 2] = vx[x + q]
                const float *vyr = st + G::S_VY + so;                        // vy rows y-2 .. y+1
                const float4 ym2 = lds4(vyr), ym1 = lds4(vyr + G::ROW), yc = lds4(vyr + 2 * G::ROW),
                             yp1 = lds4(vyr + 3 * G::ROW);
                const float4 a1 = lds4(st + G::S_A1 + so), k1 = lds4(st + G::S_K1 + so);
                const bool img = IMG >= 1 && own && zp >= zs && zp < ze;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int x = gx0 + q;
                    if (x < 2 || x >= g.Nx - 2) continue;
                    const float dvx = d4(xs[q + 2], xs[q + 1], xs[q + 3], xs[q]);
                    const float dvy = d4(at(yc, q), at(ym1, q), at(yp1, q), at(ym2, q));
                    const float dvz = d4(at(vzq[2], q), at(vzq[1], q), at(vzq[3], q), at(vzq[0], q));
                    const float sum = __fadd_rn(__fadd_rn(dvx, dvy), dvz);
                    at(p, q) = __fsub_rn(__fmul_rn(__fsub_rn(1.f, at(k1, q)), at(p, q)), __fmul_rn(at(a1, q), sum));
                    if (img) A.img_i[(long long)s * g.vol + (long long)zp * g.plane + rowo + q] = -sum;
                }
            }
        }
        if (zp == sz && src_here) {
            const int q = sx - gx0;
            if (q == 0) p.x = __fadd_rn(p.x, amp);
            else if (q == 1) p.y = __fadd_rn(p.y, amp);
            else if (q == 2) p.z = __fadd_rn(p.z, amp);
            else p.w = __fadd_rn(p.w, amp);
        }
        sts4(ring + (zp & 3) * PRF + so, p);
        if (fs_on && zp == g.fs + 1)   // p[fs-1] = -p[fs+1]; plane fs-1 is still in the ring
            sts4(ring + ((g.fs - 1) & 3) * PRF + so, make_float4(-p.x, -p.y, -p.z, -p.w));
        __syncthreads();
        // every thread is done with stage k: refill it with plane zp + 2
        if (threadIdx.x == 0 && j + 2 < n_it) issue(zp + 2, k);

        // ---- energy of the previous velocity plane, by the halo warps -------
        if (ENERGY && j >= 3) {
            f3_cluster_wait();                 // the squares of plane zv-1 are in every CTA
            if (!vwarp && j >= 4) f3_energy_reduce<TY>(A, ebuf, rank, zv - 1, y0, x0, hid);
            f3_cluster_arrive_relaxed();       // ... and read (the sums use every value read)
        }

        // ---- velocities of plane zv = zp - 2 on the tile --------------------
        if (j >= 3) {
            float4 pc = zero4(), vz = vzq[0];
            const long long o = (long long)zv * g.plane + rowo;
            if (vwarp) {
                const float *rz = ring + (zv & 3) * PRF;
                pc = lds4(rz + so);
                const float pl = __shfl_up_sync(FULL, pc.w, 1);
                const float pr1 = __shfl_down_sync(FULL, pc.x, 1), pr2 = __shfl_down_sync(FULL, pc.y, 1);
                const bool zin = zv >= g.fs && zv < g.Nz - 1;
                const bool vx_row = own && zin && y >= 1 && y < g.Ny - 1;
                const bool vy_row = own && zin && y >= 1 && y < g.Ny - 2;
                const bool vz_row = own && zv >= g.fs && zv < g.Nz - 2 && y >= 1 && y < g.Ny - 1;
                if (vx_row) {
                    const float ps[7] = {pl, pc.x, pc.y, pc.z, pc.w, pr1, pr2};   // ps[q + 1] = p[x + q]
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int x = gx0 + q;
                        if (x < 1 || x >= g.Nx - 2) continue;
                        const float dp = d4(ps[q + 2], ps[q + 1], ps[q + 3], ps[q]);
                        at(vx, q) = __fsub_rn(__fmul_rn(__fsub_rn(1.f, at(k2, q)), at(vx, q)), __fmul_rn(at(a2, q), dp));
                        if (IMG == 2) A.img_j[(long long)s * g.vol + o + q] = dp;
                    }
                }
                if (vy_row) {
                    const float4 ym1 = lds4(rz + so - G::ROW), yp1 = lds4(rz + so + G::ROW),
                                 yp2 = lds4(rz + so + 2 * G::ROW);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int x = gx0 + q;
                        if (x < 1 || x >= g.Nx - 1) continue;
                        const float dp = d4(at(yp1, q), at(pc, q), at(yp2, q), at(ym1, q));
                        at(vy, q) = __fsub_rn(__fmul_rn(__fsub_rn(1.f, at(k3, q)), at(vy, q)), __fmul_rn(at(a2, q), dp));
                        if (IMG == 2) A.img_j[((long long)g.n_shots + s) * g.vol + o + q] = dp;
                    }
                }
                if (vz_row) {
                    const float4 zm1 = lds4(ring + ((zv - 1) & 3) * PRF + so),
                                 zp1 = lds4(ring + ((zv + 1) & 3) * PRF + so),
                                 zp2 = lds4(ring + ((zv + 2) & 3) * PRF + so);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int x = gx0 + q;
                        if (x < 1 || x >= g.Nx - 1) continue;
                        const float dp = d4(at(zp1, q), at(pc, q), at(zp2, q), at(zm1, q));
                        at(vz, q) = __fsub_rn(__fmul_rn(__fsub_rn(1.f, at(k4, q)), at(vz, q)), __fmul_rn(at(a2, q), dp));
                        if (IMG == 2) A.img_j[(2LL * g.n_shots + s) * g.vol + o + q] = dp;
                    }
                }
            }
            if (ENERGY) {
                // hand the squares to the cluster before this plane's global
                // stores, so the release below waits for none of them
                f3_cluster_wait();   // every CTA of the cluster is done reading the previous squares
                if (vwarp) {
                    float *e = ebuf + ((pr - 1) * 32 + lane) * 4;
                    sts4(e, sq4(pc));
                    sts4(e + TY * 32 * 4, sq4(vx));
                    sts4(e + 2 * TY * 32 * 4, sq4(vy));
                    sts4(e + 3 * TY * 32 * 4, sq4(vz));
                    f3_cluster_arrive();
                } else {
                    f3_cluster_arrive_relaxed();
                }
            }
            if (own) {
                stg4(outS + o, pc);
                stg4(outS + g.vol + o, vx);
                stg4(outS + 2 * g.vol + o, vy);
                // vz[fs-1] = vz[fs]: the CTA of plane fs writes the mirror plane
                if (!(fs_on && zv == g.fs - 1)) stg4(outS + 3 * g.vol + o, vz);
                if (fs_on && zv == g.fs) stg4(outS + 3 * g.vol + (long long)(g.fs - 1) * g.plane + rowo, vz);
            }
        }
    }
    if (ENERGY) {
        f3_cluster_wait();
        if (!vwarp) f3_energy_reduce<TY>(A, ebuf, rank, ze - 1, y0, x0, hid);
        f3_cluster_arrive_relaxed();
        f3_cluster_wait();   // no CTA leaves while another reads its squares
    }
}

}  // namespace gb
