// Batched step kernels: one launch advances every active model of a batch
// (models of different grid size and step count, e.g. an ensemble of
// velocity particles) by one time step.  Each CTA takes one work item
// (model, tile, shot group) from a table; the per-model descriptors and TMA
// maps live in device memory.  Replaces the serial per-particle loop of
// geobrain/core/inverse.py:104-110 (one propagator call per particle).
//
// Time runs on a batch-wide clock tau.  Forward: model m is active while
// tau < nt_m, reading state level tau & 1.  Recompute of checkpoint segment
// [t0, t0 + K): model m is active while tau < min(nt_m, t_cache_m), reading
// level (tau - t0) & 1.  Adjoint: model m is active while tau < nt_m and its
// adjoint state sits in level (nt_m - 1 - tau) & 1; its imaging fields come
// from the forward's cache for tau >= t_cache_m, else from the recomputed
// segment.
#pragma once

#include "gb_adj.cuh"

namespace gb {

struct alignas(64) BatchMaps {
    CUtensorMap fld[2][3];   // forward state levels: p, vx, vz boxes
    CUtensorMap mu[2][3];    // adjoint state levels
    CUtensorMap a1, a2;      // coefficient boxes
};

struct BatchModel {
    FwdArgs f;               // forward launch template (it / out / imaging set per step)
    AdjArgs a;               // adjoint launch template (it / out / img set per step)
    float *fld[2];           // forward state levels
    float *mu[2];            // adjoint state levels
    float *cache;            // imaging cache of steps >= t_cache, or null
    float *segimg;           // imaging fields of the segment being recomputed (cache_fmt)
    long long step_img;      // elements per step of imaging fields
    int nt, t_cache, K;
    int cache_fmt;           // storage format of the cache (kImg*)
};

// Step `j` of an imaging buffer in the model's format (elements of 2, 3 or
// 4 bytes): the cache, or the recompute segment's buffer.
__device__ __forceinline__ float *img_step(const BatchModel &M, float *base, int j)
{
    const int es = M.cache_fmt == kImgBF16 ? 2 : M.cache_fmt == kImgF24 ? 3 : 4;
    return reinterpret_cast<float *>(reinterpret_cast<char *>(base) + (long long)j * M.step_img * es);
}

constexpr int kBatchForward = 0;
constexpr int kBatchRecompute = 1;

// clock: a device step counter when the launch is replayed from a CUDA graph
// (tau then counts from it: *clock + tau forward, *clock - tau in the
// adjoint), or null.
template <int R, int TZ, bool FS, bool ENERGY, int IMG>
__global__ void __launch_bounds__(NTHR, TZ <= 16 ? 2 : 1)
fwd_batch_kernel(const int4 *__restrict__ items, const BatchModel *__restrict__ models,
                 const BatchMaps *__restrict__ maps, int tau, int mode, int t0, const int *clock)
{
    if (clock) tau += *reinterpret_cast<const volatile int *>(clock);
    const int4 item = items[blockIdx.x];   // (model, tile, group, 0)
    const BatchModel &M = models[item.x];
    const int t_end = mode == kBatchForward ? M.nt : min(M.nt, M.t_cache);
    if (tau >= t_end) return;              // uniform per CTA
    const int par = mode == kBatchForward ? (tau & 1) : ((tau - t0) & 1);
    __shared__ FwdArgs A;
    if (threadIdx.x == 0) {
        A = M.f;
        A.it = tau;
        A.out = M.fld[par ^ 1];
        if (mode == kBatchForward) {
            A.imaging = (M.cache && tau >= M.t_cache) ? img_step(M, M.cache, tau - M.t_cache) : nullptr;
            A.img_fmt = M.cache_fmt;
        } else {
            A.imaging = img_step(M, M.segimg, tau - t0);
            A.img_fmt = M.cache_fmt;
            A.energy = nullptr;
            A.tr_p = A.tr_vx = A.tr_vz = nullptr;
        }
    }
    __syncthreads();
    const BatchMaps &mp = maps[item.x];
    const int s0 = item.z * A.g.shots_per_cta;
    fwd_body<R, TZ, FS, ENERGY, IMG>(&mp.fld[par][0], &mp.fld[par][1], &mp.fld[par][2], &mp.a1, &mp.a2, A, item.y, s0,
                                     min(A.g.n_shots - s0, A.g.shots_per_cta));
}

// IMGF: the imaging format every model of the batch stores (kImg*), or -1
// to read each model's at run time.
template <int R, int TZ, bool FS, bool RHO, int IMGF>
__global__ void __launch_bounds__(NTHR, TZ <= 16 ? 2 : 1)
adj_batch_kernel(const int4 *__restrict__ items, const BatchModel *__restrict__ models,
                 const BatchMaps *__restrict__ maps, int tau, const int *clock)
{
    if (clock) tau = *reinterpret_cast<const volatile int *>(clock) - tau;
    const int4 item = items[blockIdx.x];
    const BatchModel &M = models[item.x];
    if (tau >= M.nt) return;
    const int par = (M.nt - 1 - tau) & 1;
    __shared__ AdjArgs A;
    if (threadIdx.x == 0) {
        A = M.a;
        A.it = tau;
        A.out = M.mu[par ^ 1];
        const bool cached = M.cache && tau >= M.t_cache;
        A.img = cached ? img_step(M, M.cache, tau - M.t_cache) : img_step(M, M.segimg, tau - (tau / M.K) * M.K);
        A.img_fmt = M.cache_fmt;
    }
    __syncthreads();
    const BatchMaps &mp = maps[item.x];
    adj_body<R, TZ, FS, RHO, IMGF>(&mp.mu[par][0], &mp.mu[par][1], &mp.mu[par][2], &mp.a1, &mp.a2, A, item.z, item.y);
}

}  // namespace gb
