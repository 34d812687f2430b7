/*
 * geobrain_b200 — C ABI of the B200 (sm_100a) 2D acoustic propagator.
 *
 * Plain pointers, sizes and a CUDA stream; no framework types.  Every entry
 * point returns 0 on success or a negative GB_E* code; gb_last_error() gives
 * the message of the last failure on the calling thread.
 *
 * Reference interfaces these replace (paths inside the GeoBrain source tree):
 *   geobrain/physics/wave/kernels/acoustic_2d.py:294-317  acoustic_forward_kernel(...)
 *       -> gb_plan_create + gb_forward (traces, energy maps, snapshots)
 *   geobrain/physics/wave/kernels/acoustic_2d.py:448-460  torch.utils.checkpoint
 *       segments + autograd backward through acoustic_step_forward (:123-291)
 *       -> gb_forward with checkpoints + gb_backward (hand-written adjoint)
 *   geobrain/physics/wave/kernels/acoustic_2d.py:18-66     pad_model and its
 *       autograd adjoint -> done inside gb_forward / gb_backward
 *   geobrain/core/inverse.py:104-110 serial per-particle forward_fn loop
 *       -> gb_batch_* (many models, one launch per step)
 *
 * Grid conventions follow the reference: models are (nz, nx) row-major,
 * padded by nabc cells on every side to (Nz, Nx) = (nz + 2 nabc, nx + 2 nabc);
 * source and receiver positions are unpadded integer grid indices; traces are
 * (n_shots, nt, n_rcv); energy maps are (nz, nx).
 */
#ifndef GEOBRAIN_B200_H
#define GEOBRAIN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GB_OK              0
#define GB_E_ARG          -1   /* invalid argument (sizes, positions, CFL, ...) */
#define GB_E_CUDA         -2   /* a CUDA runtime call failed */
#define GB_E_WORKSPACE    -3   /* workspace too small */
#define GB_E_TIMEOUT      -4   /* a device-side bounded wait gave up */
#define GB_E_UNSUPPORTED  -5   /* option not built into this library */

/* One velocity model and its acquisition (acoustic_forward_kernel arguments
 * nx, nz, dx, dz, nt, dt, nabc, free_surface, src_n, rcv_n; half = stencil
 * half-width: 2 for the reference's 4th-order scheme, 4 for 8th order). */
typedef struct gb_model_desc {
    int32_t nz, nx, nabc, nt;
    int32_t n_shots, n_rcv, half, free_surface;
    float dt, dx;
} gb_model_desc;

/* Snapshot (checkpoint) storage formats for the gradient. */
#define GB_CKPT_F32   0
#define GB_CKPT_BF16  1   /* bf16 with one fp32 scale per (checkpoint, shot, field) */
#define GB_CKPT_F16   2   /* fp16 with one fp32 scale per (checkpoint, shot, field) */
#define GB_CKPT_F24   3   /* upper 24 bits of the fp32 (15-bit mantissa, fp32 exponent,
                             no scale), 3 bytes per value */

/* Storage formats of the imaging cache.  Both short formats keep the fp32
 * exponent (no scale) and round to nearest even:
 *   GB_IMG_BF16  16 bits (8-bit mantissa);
 *   GB_IMG_F24   24 bits (15-bit mantissa), 3 bytes per value. */
#define GB_IMG_F32   0
#define GB_IMG_BF16  1
#define GB_IMG_F24   3

/* What the forward keeps for a later gb_backward (replaces the
 * torch.utils.checkpoint segments of acoustic_2d.py:430,448-460):
 *   checkpoints       full state every checkpoint_every steps, in `format`,
 *                     gb_plan_checkpoint_bytes(plan, checkpoint_every, format)
 *                     bytes (may be NULL when cached_steps == nt);
 *   imaging           the imaging fields of the last cached_steps time steps,
 *                     gb_plan_imaging_bytes(plan, cached_steps, with_rho,
 *                     imaging_format) bytes (may be NULL when
 *                     cached_steps == 0); those steps need no recompute in
 *                     the backward;
 *   with_rho          keep / compute the fields the density gradient needs;
 *   imaging_format    GB_IMG_F32, GB_IMG_F24 or GB_IMG_BF16.  The fields
 *                     are only multiplied into the gradient sums, so each
 *                     rounding error enters the gradient once and is not
 *                     propagated by the wave equation; the sums cancel
 *                     heavily, though, so the gradient's relative error is
 *                     of the order of the format's precision (about 3e-3
 *                     for bf16, 1e-5 for f24). */
typedef struct gb_grad_store {
    void *checkpoints;
    int32_t checkpoint_every;
    int32_t format;
    void *imaging;
    int32_t cached_steps;
    int32_t with_rho;
    int32_t imaging_format;
} gb_grad_store;

typedef struct gb_plan gb_plan;   /* opaque */

/* Build a plan for one model: validates sizes and positions (host arrays of
 * unpadded indices, like the reference's src_x/src_z/rcv_x/rcv_z), bins the
 * receivers by tile and sizes the device workspace.  Replaces the set-up half
 * of acoustic_forward_kernel (acoustic_2d.py:365-420). */
int gb_plan_create(const gb_model_desc *desc,
                   const int64_t *src_x, const int64_t *src_z,
                   const int64_t *rcv_x, const int64_t *rcv_z,
                   gb_plan **out);
void gb_plan_destroy(gb_plan *plan);

/* Tile height (rows per CTA, 16 or 32) and shots per CTA; 0 keeps the
 * default.  Used by the autotuner. */
int gb_plan_set_tiling(gb_plan *plan, int tile_rows, int shots_per_cta);

/* Plain forward (gb_forward without a gradient store) as replays of one
 * CUDA graph of `steps` time steps (even, at most 64; 0 = one launch per
 * step and group; 16 by default).  The same chunk length drives the graphs
 * of the gradient (the forward steps that keep their imaging fields and the
 * adjoint steps over them) and of the batched forward and adjoint; each of
 * those graphs is captured on the first call and kept while the buffers are
 * the same.  The graph holds the step kernels of every shot group,
 * with their fork and join, and a step-counter update.  It is captured on
 * the first call, kept on the plan and replayed nt / steps times; the
 * remaining steps launch one by one.  A call with other buffers (workspace,
 * wavelet or trace pointers) captures it again. */
int gb_plan_set_graph_steps(gb_plan *plan, int steps);

/* Order of the tile kernels' CTAs in a time step.  mode 0 (default):
 * tile-major blockIdx order, one CTA per (tile, shot group).  mode 1: the
 * tiles that take the masked, damped path (those reaching into the
 * absorbing frame, the free surface or past the grid's edge) are dispatched
 * first, and the forward's last items, as many as there are resident CTAs,
 * are split into two halves of their shots, so a step ends on short items
 * (measured on the 400 x 1200, 32-shot gradient: no faster).  The results
 * are the same either way; energy sums are atomic in both. */
int gb_plan_set_schedule(gb_plan *plan, int mode);

/* The forward work list that schedule mode 1 builds for `slots` resident
 * CTAs (no device call).  config g < n_groups: the launch of shot group g
 * alone (group streams); config n_groups: one launch of every group.
 * Writes *n_items, and, when items is not NULL (cap >= *n_items), the items
 * as (tile, first shot, shots) triples. */
int gb_plan_schedule_items(gb_plan *plan, int slots, int config, int32_t *items, int cap, int *n_items);

/* Autotuner.  Times `steps` plain forward steps of this plan (no traces, no
 * energy) for each launch configuration:
 *   - tile rows 16 / 32;
 *   - shots per CTA automatic, 1, 2, 4, 8 or 16;
 *   - per-group streams on / off;
 *   - graph chunks of 16 steps or none;
 *   - the streaming forward kernel or the tile kernel.
 * It keeps the fastest on the plan and reports its time per step.  Each
 * candidate runs three times; the first is a warm-up.  The workspace must
 * hold gb_plan_autotune_workspace_bytes(plan); candidates that do not fit
 * are skipped.  Blocks until done. */
size_t gb_plan_autotune_workspace_bytes(gb_plan *plan);

/* The launch configuration in use (what the autotuner chose): tile rows,
 * effective shots per CTA, per-group streams, graph chunk steps, and the
 * streaming kernel's chunks per z-segment (0 when the tile kernel runs). */
int gb_plan_get_config(const gb_plan *plan, int *tile_rows, int *shots_per_cta, int *group_streams,
                       int *graph_steps, int *stream_chunks);

/* Forward (and recompute) steps by the streaming kernel: one CTA walks a
 * 120-column strip of one shot down a z-segment of seg_chunks 16-row chunks
 * (0 = automatic), keeping the rows it has in shared-memory rings, so that
 * each pressure row is updated once instead of once per tile plus a halo.
 * Same results as the tile kernel, bit for bit.  Used when enabled, the
 * tiles are 16 rows and the model has no free surface; otherwise the tile
 * kernel runs.  Off by default; the autotuner tries it. */
int gb_plan_set_streaming(gb_plan *plan, int enable, int seg_chunks);

/* Absorbing layers.  GB_ABSORB_DAMPING (default) is the reference's
 * damping PML, driven by the damp array (boundary/pml.py).
 * GB_ABSORB_CPML is an opt-in convolutional PML with memory variables, an
 * extension the reference does not have; the damp array is not used:
 *   - per axis, a quadratic profile d = d0 (depth / nabc)^2 with
 *     d0 = -3 vmax ln(1e-6) / (2 nabc dx), on both sides (not above a free
 *     surface); b = exp(-d dt), a = b - 1, at integer and half points;
 *   - every derivative g entering an update becomes g + psi, with
 *     psi' = b psi + a g (psi_px, psi_pz for p; psi_vx, psi_vz for the
 *     velocities), and the k damping terms are dropped.
 * Gradients: gb_backward runs the CPML adjoint, which reads every step's
 * imaging fields from the store (cached_steps = nt; otherwise
 * GB_E_UNSUPPORTED), so the memory variables need no checkpoints.  Batched
 * runs reject CPML plans; the streaming kernel is not used with it. */
#define GB_ABSORB_DAMPING 0
#define GB_ABSORB_CPML    1
int gb_plan_set_absorbing(gb_plan *plan, int mode, float vmax);
int gb_plan_autotune(gb_plan *plan, const float *vp, const float *rho, const float *damp,
                     const float *wavelet, void *workspace, size_t workspace_bytes, int32_t steps,
                     void *stream, float *best_ms_per_step);

/* Resident forward (plain gb_forward without a store, damping layers only):
 * one launch runs many time steps, each CTA keeping a 120-column x
 * tile_rows tile of one shot, plus its halo, in shared memory.  The thread
 * that updates a cell next to a tile edge sends it to the neighbouring
 * tile, and the rest of the tile is updated while it travels.
 * It is the plain forward's fast path when a step is too small to fill the
 * GPU: few shots, or a small grid.  The traces are those of the tile kernel,
 * bit for bit.  mode: -1 automatic (the default: on when every shot's tiles
 * fit on the device's SMs at once, one CTA per SM, with the exchange through
 * global memory after each half-step and the smallest tile height that
 * fits), 0 off, 1 on with the exchange
 * through global memory (a cooperative launch; each float travels as an
 * 8-byte (value, tag) word the receiver polls, bounded; shots beyond one
 * launch run in further launches), 2 on with the exchange through
 * distributed shared memory: one thread-block cluster of at most 16 CTAs per
 * shot, the sender storing into the neighbour's halo, hardware cluster
 * barriers in place of the tags; 3 on with one exchange a step through
 * global memory, each tile also updating p on R rows and columns of its
 * neighbours' cells from the same inputs (4th order without a free surface
 * only).
 * tile_rows: 4, 8, 12, 16, 24, 32, 36 or 40, or 0 for the smallest that
 * fits.  With a free surface, rows fs-1 .. fs+1 must fall in one tile.
 * GB_E_UNSUPPORTED when mode 1 finds no tiling (or the plan uses CPML); the
 * plan then stays automatic.  The workspace (gb_plan_workspace_bytes) grows
 * by the exchange strips. */
int gb_plan_set_resident(gb_plan *plan, int mode, int tile_rows);
/* Tile rows of the resident forward in use (0: the tile kernel runs),
 * shots per launch, and the exchange: 0 through global memory after each
 * half-step, 1 through distributed shared memory, 2 once a step through
 * global memory.  Any pointer may be NULL. */
int gb_plan_get_resident(const gb_plan *plan, int *tile_rows, int *shots_per_launch, int *cluster);

/* Run each group of shots on its own stream (forked from and joined back to
 * the caller's stream; on by default).  Groups never interact, so their
 * kernels fill each other's tails. */
int gb_plan_set_group_streams(gb_plan *plan, int enable);

/* Bytes of device workspace gb_forward / gb_backward need.  with_gradient:
 * 0 forward only; 1 adds the adjoint state, the imaging buffer of one
 * checkpoint segment and the velocity-gradient sums; 2 also the density
 * gradient's.  The workspace is used from its first 256-byte boundary. */
size_t gb_plan_workspace_bytes(const gb_plan *plan, int with_gradient, int checkpoint_every);

/* The exact workspace gb_backward needs for a store: its recompute segment
 * buffer holds segment_steps = max(1, min(checkpoint_every, nt -
 * cached_steps)) steps of imaging fields in the store's imaging_format (the
 * recomputed fields are rounded like the cached ones).  gb_plan_workspace_bytes
 * with with_gradient > 0 is the fp32 upper bound of it. */
size_t gb_plan_gradient_workspace_bytes(const gb_plan *plan, int with_rho, int segment_steps,
                                        int imaging_format);

/* Bytes of checkpoint storage for a given segment length and format (0 for
 * an unknown format). */
size_t gb_plan_checkpoint_bytes(const gb_plan *plan, int checkpoint_every, int ckpt_format);

/* Bytes of the imaging cache for the last cached_steps time steps
 * (imaging_format one of GB_IMG_*; 0 for an unknown format). */
size_t gb_plan_imaging_bytes(const gb_plan *plan, int cached_steps, int with_rho, int imaging_format);

/* Forward modelling, all nt steps, on `stream` (acoustic_forward_kernel,
 * acoustic_2d.py:294-501).  Device pointers:
 *   vp, rho   (nz, nx) float32       damp (Nz, Nx) float32
 *   wavelet   (n_shots, nt) float32  (the source adds dt * wavelet[s, it])
 *   trace_p / trace_vx / trace_vz (n_shots, nt, n_rcv) float32, each may be NULL
 *   energy_p / energy_vx / energy_vz (nz, nx) float32, NULL skips the energy sums
 *   snapshots ((nt + snapshot_every - 1) / snapshot_every, nz, nx) float32,
 *             pressure of shot 0 at the end of each snapshot chunk, or NULL
 *   store     NULL for plain modelling, or what to keep for gb_backward.
 */
int gb_forward(gb_plan *plan, const float *vp, const float *rho, const float *damp,
               const float *wavelet,
               float *trace_p, float *trace_vx, float *trace_vz,
               float *energy_p, float *energy_vx, float *energy_vz,
               int32_t snapshot_every, float *snapshots, const gb_grad_store *store,
               void *workspace, size_t workspace_bytes, void *stream);

/* Gradient of a loss L with respect to vp and rho, given the adjoint sources
 * res_* = dL/d(trace_*) (n_shots, nt, n_rcv) float32 (any may be NULL), and
 * the store a gb_forward call with the same plan and model filled.  Runs the
 * hand-written adjoint backwards in time with the zero-lag imaging condition
 * fused in: over the cached steps first, then one checkpoint segment at a
 * time after an fp32 recompute of that segment from its checkpoint.  Sums
 * over shots and time with compensated fp32 summation and folds the padding
 * back into the edge cells (the adjoint of pad_model).  grad_vp / grad_rho
 * are (nz, nx) float32 and are overwritten; grad_rho may be NULL (it needs a
 * store made with with_rho).  grad_wavelet, (n_shots, nt) float32 or NULL,
 * receives dL/d(wavelet), what autograd through the reference's source
 * injection gives (acoustic_2d.py:228-237); it needs every source inside the
 * pressure update region (padded z in [max(fs+1, R), Nz-1-R], x in
 * [R, Nx-1-R]; GB_E_UNSUPPORTED otherwise).  Workspace: gb_plan_gradient_workspace_bytes
 * (the recompute segments only cover the uncached steps, and their imaging
 * fields are kept in the store's imaging_format). */
int gb_backward(gb_plan *plan, const float *vp, const float *rho, const float *damp,
                const float *wavelet,
                const float *res_p, const float *res_vx, const float *res_vz,
                const gb_grad_store *store,
                float *grad_vp, float *grad_rho, float *grad_wavelet,
                void *workspace, size_t workspace_bytes, void *stream);

/* Profiling (used by the benchmark): when enabled, gb_forward and
 * gb_backward record CUDA events on their stream around the forward loop,
 * each segment's fp32 recompute and each adjoint sweep, and count their
 * kernel launches and time steps.  gb_plan_profile waits for those events,
 * returns the summed milliseconds per phase, the launch count and the time
 * steps per phase (forward, recompute, adjoint; array of 3) since the last
 * call, and resets them.  Any output pointer may be NULL. */
int gb_plan_set_profiling(gb_plan *plan, int enable);
/* Host-side launch calls (step-kernel launches and CUDA graph replays) since
 * profiling was last enabled; gb_plan_profile does not reset it.  The plain
 * forward, the gradient's forward and adjoint over the steps whose imaging
 * fields the forward kept, and the batched forward and adjoint run in
 * chunks of gb_plan_set_graph_steps steps replayed from CUDA graphs, so
 * this is about that many times smaller than the kernel launch count. */
int gb_plan_launch_calls(const gb_plan *plan, long long *calls);
int gb_plan_profile(gb_plan *plan, double *ms_forward, double *ms_recompute, double *ms_adjoint,
                    long long *launches, long long *phase_steps);

/* Batches of models (velocity particles of one ensemble, or unrelated models
 * of uneven size and step count).  Every plan of a batch uses one stencil
 * order, one free-surface setting and 16-row tiles; a gradient batch shares
 * checkpoint_every, snapshot format and with_rho.  Each model keeps its own
 * workspace (gb_plan_workspace_bytes as for the single-model calls) and
 * outputs; the batch workspace holds the per-model descriptors and the work
 * list.  One kernel launch per time step advances every model still running
 * (replaces the serial per-particle forward_fn loop of
 * geobrain/core/inverse.py:104-110). */
typedef struct gb_model_io {
    const float *vp, *rho, *damp, *wavelet;         /* as gb_forward */
    float *trace_p, *trace_vx, *trace_vz;           /* forward outputs (may be NULL) */
    float *energy_p, *energy_vx, *energy_vz;        /* forward outputs (may be NULL) */
    const float *res_p, *res_vx, *res_vz;           /* backward inputs (may be NULL) */
    float *grad_vp, *grad_rho;                      /* backward outputs */
    const gb_grad_store *store;                     /* what the forward keeps (NULL: plain modelling) */
    void *workspace;                                /* this model's workspace */
    size_t workspace_bytes;
} gb_model_io;

size_t gb_batch_workspace_bytes(gb_plan *const *plans, int n_models);
int gb_batch_forward(gb_plan *const *plans, int n_models, const gb_model_io *io,
                     void *batch_workspace, size_t batch_workspace_bytes, void *stream);
int gb_batch_backward(gb_plan *const *plans, int n_models, const gb_model_io *io,
                      void *batch_workspace, size_t batch_workspace_bytes, void *stream);

/* Trace-normalised L2 misfit and its adjoint source, on the device.  It
 * replaces the misfit of examples/09_acoustic_fwi.py:290-319:
 * normalize_traces, per_trace_l2, active_mask.  For pred and obs of shape
 * (n_shots, nt, n_rcv), float32:
 *   - each trace is divided by its max |value| (clamped to 1e-30);
 *   - the per-trace L2 norm of obs_n - pred_n is summed over the traces
 *     that are not silent in both.
 * Outputs:
 *   - loss: one float32 on the device, summed in fp64 in a fixed order;
 *   - per_trace: (n_shots, n_rcv) float32, the L_j, 0 for silent traces;
 *   - adj: same shape as pred, may be NULL; d loss / d pred, including the
 *     gradient of each trace's max.  It is the residual gb_backward takes.
 *     Silent traces and traces with L_j = 0 get zeros; autograd through the
 *     example's expression gives NaN there. */
int gb_trace_misfit(const float *pred, const float *obs, int32_t n_shots, int32_t nt, int32_t n_rcv,
                    float *adj, float *per_trace, float *loss, void *stream);

/* Synchronises `stream` and reports the device-side status word of a
 * workspace after gb_forward / gb_backward: GB_OK, or GB_E_TIMEOUT if a
 * bounded wait inside a kernel gave up. */
int gb_workspace_status(const void *workspace, void *stream);

/* Failure-detection self-test of the bounded waits (no counterpart in the
 * reference).  One CTA waits on an mbarrier that completes only if
 * `complete` is nonzero.  Otherwise the wait gives up after max_polls polls
 * (1 .. 2^22; the step kernels use 2^22) and sets the workspace status word, as a
 * step kernel does when its loads never land.  Returns what
 * gb_workspace_status then reads: GB_OK, or GB_E_TIMEOUT.  No GPU fault and
 * no hang either way; the context stays usable.  Workspace: 4 bytes past
 * the first 256-byte boundary (as every other workspace here). */
int gb_selftest_bounded_wait(void *workspace, size_t workspace_bytes, int32_t complete, int32_t max_polls,
                             void *stream);

/* Forward modelling without any device allocation: the same computation and
 * outputs as gb_forward (no checkpoints), with the scratch held in a static
 * device array inside this library instead of a caller workspace.
 * No counterpart in the reference.  It is meant for callers that cannot
 * allocate device memory (a host whose memory pool owns the GPU and offers
 * no allocation hook).  Limits and behaviour:
 *   - the array is gb_static_scratch_bytes() (64 MiB) on every GPU that
 *     loads the library, held until the process exits; a model whose
 *     scratch (gb_plan_workspace_bytes(plan, 0, 0) less its 256 bytes of
 *     alignment slack, which the aligned array does not need) exceeds it is
 *     rejected with GB_E_WORKSPACE;
 *   - the first call on each device and CUDA context looks the array's
 *     device address up (cudaGetSymbolAddress) with that device current, so
 *     a new context (after cudaDeviceReset, or one the host created) gets
 *     its own module's address; make that first call before any stream
 *     capture;
 *   - every call shares the one array per device: calls whose work overlaps
 *     on the GPU (other streams, other threads) race and corrupt each other;
 *   - it calls no cudaMalloc / cudaFree; inputs and outputs are the caller's;
 *   - it launches one kernel per step and shot group, whatever
 *     gb_plan_set_graph_steps says (instantiating a graph allocates). */
size_t gb_static_scratch_bytes(void);
int gb_forward_static_scratch(gb_plan *plan, const float *vp, const float *rho, const float *damp,
                              const float *wavelet,
                              float *trace_p, float *trace_vx, float *trace_vz,
                              float *energy_p, float *energy_vx, float *energy_vz,
                              int32_t snapshot_every, float *snapshots, void *stream);

/* ---------------------------------------------------------------------
 * 3-D acoustic forward modelling (4th order), a drop-in for
 * acoustic_forward_kernel_3d (geobrain/physics/wave/kernels/acoustic_3d.py
 * :303-476): padding, coefficients and every time step on the device.
 * -------------------------------------------------------------------- */
typedef struct gb3_model_desc {
    int32_t nz, ny, nx, nabc, nt;
    int32_t n_shots, n_rcv, free_surface;
    float dt, dx, dy, dz;      /* the reference scales every derivative by 1/dz */
} gb3_model_desc;

size_t gb3_workspace_bytes(const gb3_model_desc *desc);

/* vp, rho: (nz, ny, nx); damp: (nz+2nabc, ny+2nabc, nx+2nabc); wavelet:
 * (n_shots, nt); positions: host int64 arrays of unpadded indices.  A source
 * may sit anywhere in the padded grid; a receiver must lie where vx, vy and
 * vz exist (padded index <= N-2 on each axis), since all four fields are
 * recorded.  Traces: (n_shots, nt, n_rcv), any may be NULL.  Energies:
 * (nz, ny, nx), all four or none (overwritten).  Device pointers;
 * asynchronous on `stream`. */
int gb3_forward(const gb3_model_desc *desc, const int64_t *src_x, const int64_t *src_y, const int64_t *src_z,
                const int64_t *rcv_x, const int64_t *rcv_y, const int64_t *rcv_z,
                const float *vp, const float *rho, const float *damp, const float *wavelet,
                float *trace_p, float *trace_vx, float *trace_vy, float *trace_vz,
                float *energy_p, float *energy_vx, float *energy_vy, float *energy_vz,
                float *checkpoints, int32_t checkpoint_every, float *imaging, int32_t imaging_rho,
                void *workspace, size_t workspace_bytes, void *stream);

/* Gradient of the 3-D path (the reference differentiates it with autograd
 * through torch.utils.checkpoint, acoustic_3d.py:446-460).  The forward keeps
 * what the adjoint needs in one of two ways:
 *   - checkpoints: the full state before every checkpoint_every-th step
 *     (gb3_checkpoint_bytes); gb3_backward recomputes each segment from its
 *     checkpoint, keeping the imaging fields;
 *   - imaging (no recompute): every step's imaging fields, I = -div v (and,
 *     with imaging_rho, dp/dx, dp/dy, dp/dz), gb3_imaging_bytes(desc,
 *     imaging_rho) bytes, [nt][1 or 4][n_shots][vol] fp32.
 * Either (or both) may be NULL in gb3_forward when no gradient follows.
 * gb3_backward takes the imaging buffer if it is not NULL (checkpoints may
 * then be NULL; grad_rho needs imaging_rho), else the checkpoints, and runs
 * the exact discrete adjoint backwards in time with the zero-lag imaging
 * condition.  res_* = dL/d(trace_*) (n_shots, nt, n_rcv), any may be NULL.
 * grad_vp, grad_rho: (nz, ny, nx), overwritten; grad_rho may be NULL.
 * grad_wavelet: (n_shots, nt) or NULL, receives dL/d(wavelet) (what
 * autograd through the reference's source line gives, acoustic_3d.py:153-163;
 * any source position).
 * Workspace: gb3_backward_workspace_bytes(desc, checkpoint_every,
 * grad_rho != NULL), with checkpoint_every = 0 for the imaging buffer. */
size_t gb3_checkpoint_bytes(const gb3_model_desc *desc, int32_t checkpoint_every);
size_t gb3_imaging_bytes(const gb3_model_desc *desc, int32_t with_rho);
size_t gb3_backward_workspace_bytes(const gb3_model_desc *desc, int32_t checkpoint_every, int32_t with_rho);
int gb3_backward(const gb3_model_desc *desc, const int64_t *src_x, const int64_t *src_y, const int64_t *src_z,
                 const int64_t *rcv_x, const int64_t *rcv_y, const int64_t *rcv_z,
                 const float *vp, const float *rho, const float *damp, const float *wavelet,
                 const float *res_p, const float *res_vx, const float *res_vy, const float *res_vz,
                 const float *checkpoints, int32_t checkpoint_every, const float *imaging,
                 int32_t imaging_rho, float *grad_vp, float *grad_rho, float *grad_wavelet,
                 void *workspace, size_t workspace_bytes, void *stream);

/* Selects the 3-D step kernels, process-wide (default 0):
 *   1, 2  one fused launch per time step (per 8 shots when energy maps
 *      are asked for): pressure, source, mirrors and velocities of a
 *      z-chunk, TMA-staged, in tiles of 8 (1) or 16 (2) rows, the state
 *      alternating between two workspace buffers;
 *   0  the split pressure and velocity kernels, one state updated in place
 *      (the faster: 93 against 25 Gcell-updates/s measured on a 200^3 model
 *      with a 20-cell PML and 4 shots).
 * Both give bit-identical traces, energies, states and gradients.  The
 * workspace sizes above follow the setting in force when they are asked
 * for.  Returns the previous setting.  gb_workspace_status reads the device
 * status word of a 3-D workspace as of a 2-D one. */
int gb3_set_fused_step(int32_t on);

/* Message of the last failure on this thread ("" if none). */
const char *gb_last_error(void);

/* Library version string. */
const char *gb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* GEOBRAIN_B200_H */
