// Host-side handles of the step kernel variants.  Each family is instantiated
// in its own translation unit (gb_pick_*.cu), so that the build compiles the
// template variants in parallel; gb_capi.cu launches them through these
// handles (a kernel's host stub works from any translation unit).
#pragma once

#include <cstddef>

namespace gb {
namespace host {

struct StepKernel {
    void *fn = nullptr;
    size_t smem = 0;
    bool stream = false;    // fwd_stream_kernel: launched over (strip, segment, shot)
};

// fwd_step_kernel<R, TZ, FS, ENERGY, IMG> (gb_fwd.cuh); fn is null for an
// unsupported combination.  gb_pick_fwd2.cu / gb_pick_fwd4.cu.
StepKernel fwd_tile_kernel_r2(int tz, bool fs, bool en, int img);
StepKernel fwd_tile_kernel_r4(int tz, bool fs, bool en, int img);
// fwd_stream_kernel<R, ENERGY, IMG> (gb_stream.cuh).  gb_pick_stream.cu.
StepKernel fwd_stream_kernel_for(int R, bool en, int img);
// adj_step_kernel<R, TZ, FS, RHO, IMGF> (gb_adj.cuh).  gb_pick_adj2.cu / gb_pick_adj4.cu.
StepKernel adj_tile_kernel_r2(int tz, bool fs, bool rho, int img_fmt);
StepKernel adj_tile_kernel_r4(int tz, bool fs, bool rho, int img_fmt);
// fwd_batch_kernel / adj_batch_kernel (gb_batch.cuh), 16-row tiles.  gb_pick_batch.cu.
StepKernel fwd_batch_kernel_for(int R, bool fs, bool en, int img);
// imgf: the imaging format all models of the batch store, or -1 (per model)
StepKernel adj_batch_kernel_for(int R, bool fs, bool rho, int imgf);

}  // namespace host
}  // namespace gb

namespace gb {
namespace host {

// resident_fwd_kernel<R, NW, TZ> (gb_resident.cuh) for the tile heights in
// kResidentRows; fn is null for other heights.  gb_pick_resident.cu.
constexpr int kResidentRows[] = {4, 8, 12, 16, 24, 32, 36, 40};
struct ResidentKernel {
    void *fn = nullptr;
    size_t smem = 0;
    int threads = 0;
    size_t tile_words = 0;      // 8-byte (value, tag) exchange words per tile
};
// exchange: 0 through global memory after the p and the v updates; 1 through
// distributed shared memory within one thread-block cluster per shot (tiles
// of a shot <= 16); 2 through global memory once per step, p also updated on
// the neighbours' edge rows and columns (gb_resident_sx.cuh: 4th order, no
// free surface).
ResidentKernel resident_kernel(int R, int tz, int exchange);

}  // namespace host
}  // namespace gb
