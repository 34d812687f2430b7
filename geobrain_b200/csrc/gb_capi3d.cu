// C ABI of the 3-D acoustic path (declared in include/geobrain_b200.h):
// workspace layouts, positions and the host-side time loops that drive the
// kernels of gb_3d.cuh.
#include "gb_host.h"

#include "gb_3d.cuh"
#include "gb_3d_fused.cuh"

#include <algorithm>
#include <atomic>
#include <string>
#include <vector>

using namespace gb;
using gb::host::align256;
using gb::host::aligned_ws;
using gb::host::fail;

namespace {

// 1 / 2: one step3_fused_kernel launch per step (per 8 shots with energy
// maps) with tiles of 8 / 16 rows, the state ping-ponging between two
// buffers; 0 (default): p3_kernel + v3_kernel in place, the faster as
// measured.  Each call reads it once: its layout and its kernels agree.
std::atomic<int> g_step3_fused{0};

using F3Fn = void (*)(const CUtensorMap, const CUtensorMap, const CUtensorMap, const Fused3Args);

// What the host needs of one tile height of the fused step.
struct F3Shape {
    int rows, pr, yr, threads;
    size_t smem;
    F3Fn fn[2][3];   // [energy][imaging fields]
};

template <int TY>
F3Shape f3_shape()
{
    using G = F3Geo<TY>;
    return F3Shape{TY, G::PR, G::YR, G::NT, G::SMEM,
                   {{step3_fused_kernel<TY, false, 0>, step3_fused_kernel<TY, false, 1>,
                     step3_fused_kernel<TY, false, 2>},
                    {step3_fused_kernel<TY, true, 0>, step3_fused_kernel<TY, true, 1>,
                     step3_fused_kernel<TY, true, 2>}}};
}

const F3Shape &f3_shape_of(int mode)
{
    static const F3Shape s8 = f3_shape<8>(), s16 = f3_shape<16>();
    return mode == 2 ? s16 : s8;
}

// 4-D map over n_fields volumes [n_fields][Nz][Ny][pitch] fp32; boxes of 128
// columns x box_rows rows of one plane; everything outside reads as zero.
int make_map4(CUtensorMap *map, const float *base, const Geo3 &g, int n_fields, int box_rows)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc;
    if (int rc = gb::host::tensor_map_encoder(&enc)) return rc;
    if (reinterpret_cast<uintptr_t>(base) & 15) return fail(GB_E_ARG, "3-D volume not 16-byte aligned");
    cuuint64_t dims[4] = {(cuuint64_t)g.pitch, (cuuint64_t)g.Ny, (cuuint64_t)g.Nz, (cuuint64_t)n_fields};
    cuuint64_t strides[3] = {(cuuint64_t)g.pitch * 4, (cuuint64_t)g.plane * 4, (cuuint64_t)g.vol * 4};
    cuuint32_t box[4] = {128, (cuuint32_t)box_rows, 1, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float *>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(GB_E_CUDA, "cuTensorMapEncodeTiled (4-D) failed (" + std::to_string((int)r) + ")");
    return GB_OK;
}

// The fused step's launch state: maps of both state buffers and of the
// coefficients, the tiling, and which buffer holds the current state.
struct Fused3 {
    CUtensorMap mS[2], mY[2], mC;
    float *buf[2];
    int cur;
    int tiles_x, tiles_y, chunk, n_chunks;
    const F3Shape *shape;
};

// Number of z-chunks: the launch's CTAs fill whole waves of the resident
// slots, discounted by the 3 extra pressure planes each chunk recomputes.
int f3_chunks(const Geo3 &g, int tiles, int ns, int slots)
{
    int best = 1;
    double best_eff = 0.0;
    for (int c = 1; c <= 32; ++c) {
        const int chunk = (g.Nz + c - 1) / c;
        if (chunk < 4 && c > 1) break;
        const int n = (g.Nz + chunk - 1) / chunk;
        const long long work = (long long)n * tiles * ns;
        const long long waves = (work + slots - 1) / slots;
        const double eff = (double)work / ((double)waves * slots) * chunk / (chunk + 3.0);
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best = n;
        }
    }
    return best;
}

int fused3_setup(const Geo3 &g, float *buf0, float *buf1, const float *coef, bool energy, int mode, Fused3 *F)
{
    const F3Shape &sh = f3_shape_of(mode);
    F->shape = &sh;
    F->buf[0] = buf0;
    F->buf[1] = buf1;
    F->cur = 0;
    for (int k = 0; k < 2; ++k) {
        if (int rc = make_map4(&F->mS[k], F->buf[k], g, 4 * g.n_shots, sh.pr)) return rc;
        if (int rc = make_map4(&F->mY[k], F->buf[k], g, 4 * g.n_shots, sh.yr)) return rc;
    }
    if (int rc = make_map4(&F->mC, coef, g, 6, sh.pr)) return rc;
    for (int e = 0; e < 2; ++e)
        for (int i = 0; i < 3; ++i)
            GB_CUDA(cudaFuncSetAttribute((const void *)sh.fn[e][i], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sh.smem));
    int dev = 0, sms = 0, per_sm = 0;
    GB_CUDA(cudaGetDevice(&dev));
    GB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)sh.fn[energy ? 1 : 0][0], sh.threads,
                                                          sh.smem));
    if (per_sm < 1) return fail(GB_E_UNSUPPORTED, "the fused 3-D step does not fit on this device");
    F->tiles_x = (g.Nx + TX - 1) / TX;
    F->tiles_y = (g.Ny + sh.rows - 1) / sh.rows;
    const int ns = energy ? std::min(g.n_shots, kF3MaxCluster) : g.n_shots;
    F->n_chunks = f3_chunks(g, F->tiles_x * F->tiles_y, ns, per_sm * sms);
    F->chunk = (g.Nz + F->n_chunks - 1) / F->n_chunks;
    F->n_chunks = (g.Nz + F->chunk - 1) / F->chunk;
    return GB_OK;
}

// One time step of every shot from F->buf[cur] into the other buffer; with
// energy maps the shots go in clusters of at most 8 (one launch each).
int fused3_step(const Geo3 &g, Fused3 &F, Fused3Args &A, int it, cudaStream_t st)
{
    const bool energy = A.energy[0] != nullptr;
    const int img = A.img_j ? 2 : A.img_i ? 1 : 0;
    A.g = g;
    A.it = it;
    A.tiles_x = F.tiles_x;
    A.tiles_y = F.tiles_y;
    A.chunk = F.chunk;
    A.in = F.buf[F.cur];
    A.out = F.buf[F.cur ^ 1];
    const int group = energy ? kF3MaxCluster : g.n_shots;
    for (int s0 = 0; s0 < g.n_shots; s0 += group) {
        A.shot0 = s0;
        A.ns = std::min(group, g.n_shots - s0);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(F.n_chunks * F.tiles_y * F.tiles_x * A.ns));
        cfg.blockDim = dim3(F.shape->threads);
        cfg.dynamicSmemBytes = F.shape->smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        if (energy) {
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = (unsigned)A.ns;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
        }
        void *args[] = {(void *)&F.mS[F.cur], (void *)&F.mY[F.cur], (void *)&F.mC, (void *)&A};
        GB_CUDA(cudaLaunchKernelExC(&cfg, (const void *)F.shape->fn[energy ? 1 : 0][img], args));
    }
    F.cur ^= 1;
    return GB_OK;
}

}  // namespace

extern "C" {

int gb3_set_fused_step(int32_t on)
{
    return g_step3_fused.exchange((on == 1 || on == 2) ? on : 0);
}

namespace {

// The device status word (gb_workspace_status) sits at offset 0 of both
// layouts; state2 is the second state buffer of the fused step.
struct Layout3 {
    size_t err, state, state2, coef, src, rcv, total;
};

bool geo3_of(const gb3_model_desc *d, Geo3 *g)
{
    if (!d || d->nz < 1 || d->ny < 1 || d->nx < 1 || d->nabc < 0 || d->nt < 1 || d->n_shots < 1 || d->n_rcv < 0)
        return false;
    g->nz = d->nz; g->ny = d->ny; g->nx = d->nx; g->pml = d->nabc;
    g->Nz = d->nz + 2 * d->nabc; g->Ny = d->ny + 2 * d->nabc; g->Nx = d->nx + 2 * d->nabc;
    g->pitch = (g->Nx + 31) / 32 * 32;
    g->fs = d->free_surface ? d->nabc : 1;
    g->n_shots = d->n_shots; g->nt = d->nt; g->n_rcv = d->n_rcv;
    g->dt = d->dt;
    g->plane = (long long)g->Ny * g->pitch;
    g->vol = (long long)g->Nz * g->plane;
    return true;
}

// mode: the step kernels (gb3_set_fused_step) the layout is for
Layout3 layout3(const Geo3 &g, int mode)
{
    Layout3 L{};
    size_t o = 0;
    L.err = o; o = align256(o + 4);
    L.state = o; o = align256(o + (size_t)g.n_shots * 4 * g.vol * 4);
    L.state2 = o; o = align256(o + (mode ? (size_t)g.n_shots * 4 * g.vol * 4 : 0));
    L.coef = o; o = align256(o + 6 * (size_t)g.vol * 4);
    L.src = o; o = align256(o + 3 * (size_t)g.n_shots * 4);
    L.rcv = o; o = align256(o + 3 * (size_t)std::max(g.n_rcv, 1) * 4);
    L.total = o;
    return L;
}

}  // namespace

size_t gb3_workspace_bytes(const gb3_model_desc *desc)
{
    Geo3 g;
    if (!geo3_of(desc, &g)) return 0;
    return layout3(g, g_step3_fused.load()).total + 256;
}

size_t gb3_checkpoint_bytes(const gb3_model_desc *desc, int32_t checkpoint_every)
{
    Geo3 g;
    if (!geo3_of(desc, &g) || checkpoint_every < 1) return 0;
    const size_t n_ck = (g.nt + checkpoint_every - 1) / checkpoint_every;
    return n_ck * (size_t)g.n_shots * 4 * g.vol * 4;
}

namespace {

// positions -> padded device tables; shared by the forward and the backward
int stage_positions3(const Geo3 &g, const int64_t *src_x, const int64_t *src_y, const int64_t *src_z,
                     const int64_t *rcv_x, const int64_t *rcv_y, const int64_t *rcv_z, int *d_src, int *d_rcv,
                     cudaStream_t st)
{
    if (!src_x || !src_y || !src_z) return fail(GB_E_ARG, "null source positions");
    if (g.n_rcv > 0 && (!rcv_x || !rcv_y || !rcv_z)) return fail(GB_E_ARG, "null receiver positions");
    // positions: unpadded indices, as the reference takes them (it adds nabc,
    // acoustic_3d.py:398-403); sources anywhere in the padded grid, receivers
    // where vx / vy / vz exist too (the reference indexes all four fields)
    std::vector<int> hs(3 * g.n_shots), hr(3 * std::max(g.n_rcv, 1));
    for (int s = 0; s < g.n_shots; ++s) {
        const long long z = src_z[s] + g.pml, y = src_y[s] + g.pml, x = src_x[s] + g.pml;
        if (z < 0 || z >= g.Nz || y < 0 || y >= g.Ny || x < 0 || x >= g.Nx)
            return fail(GB_E_ARG, "source " + std::to_string(s) + " lies outside the padded grid");
        hs[s] = (int)z; hs[g.n_shots + s] = (int)y; hs[2 * g.n_shots + s] = (int)x;
    }
    for (int r = 0; r < g.n_rcv; ++r) {
        const long long z = rcv_z[r] + g.pml, y = rcv_y[r] + g.pml, x = rcv_x[r] + g.pml;
        if (z < 0 || z > g.Nz - 2 || y < 0 || y > g.Ny - 2 || x < 0 || x > g.Nx - 2)
            return fail(GB_E_ARG, "receiver " + std::to_string(r) + " lies outside the velocity grids");
        hr[r] = (int)z; hr[g.n_rcv + r] = (int)y; hr[2 * g.n_rcv + r] = (int)x;
    }
    // pageable host vectors: cudaMemcpyAsync copies them before returning
    GB_CUDA(cudaMemcpyAsync(d_src, hs.data(), hs.size() * 4, cudaMemcpyHostToDevice, st));
    if (g.n_rcv) GB_CUDA(cudaMemcpyAsync(d_rcv, hr.data(), 3 * (size_t)g.n_rcv * 4, cudaMemcpyHostToDevice, st));
    return GB_OK;
}

// One forward step of every shot (optionally writing the imaging fields).
int step3(const Geo3 &g, Args3 &A, int it, bool fs, cudaStream_t st)
{
    const dim3 block(32, 4), grid((g.Nx + 127) / 128, (g.Ny + 3) / 4, g.Nz);
    A.it = it;
    p3_kernel<<<grid, block, 0, st>>>(A);
    if (fs) mirror3_kernel<<<148, 256, 0, st>>>(g, A.state, 0, 2, -1.f);
    v3_kernel<<<grid, block, 0, st>>>(A);
    if (fs) mirror3_kernel<<<148, 256, 0, st>>>(g, A.state, 3, 1, 1.f);
    GB_CUDA(cudaGetLastError());
    return GB_OK;
}

}  // namespace

int gb3_forward(const gb3_model_desc *desc, const int64_t *src_x, const int64_t *src_y, const int64_t *src_z,
                const int64_t *rcv_x, const int64_t *rcv_y, const int64_t *rcv_z, const float *vp, const float *rho,
                const float *damp, const float *wavelet, float *trace_p, float *trace_vx, float *trace_vy,
                float *trace_vz, float *energy_p, float *energy_vx, float *energy_vy, float *energy_vz,
                float *checkpoints, int32_t checkpoint_every, float *imaging, int32_t imaging_rho, void *workspace,
                size_t workspace_bytes, void *stream)
{
    gb::host::clear_error();
    Geo3 g;
    if (!geo3_of(desc, &g)) return fail(GB_E_ARG, "invalid 3-D model description");
    if (checkpoints && checkpoint_every < 1) return fail(GB_E_ARG, "checkpoint_every must be >= 1");
    if (!vp || !rho || !damp || !wavelet) return fail(GB_E_ARG, "null argument");
    if (!(desc->dt > 0.f) || !(desc->dz > 0.f)) return fail(GB_E_ARG, "dt and dz must be positive");
    if (g.Nz > 65535) return fail(GB_E_ARG, "at most 65535 padded z planes");
    const int mode = g_step3_fused.load();
    const Layout3 L = layout3(g, mode);
    char *ws = aligned_ws(workspace);
    if (!workspace || workspace_bytes < L.total + (size_t)(ws - reinterpret_cast<char *>(workspace)))
        return fail(GB_E_WORKSPACE, "workspace too small");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    float *state = reinterpret_cast<float *>(ws + L.state);
    float *state2 = reinterpret_cast<float *>(ws + L.state2);
    float *coef = reinterpret_cast<float *>(ws + L.coef);
    int *d_src = reinterpret_cast<int *>(ws + L.src), *d_rcv = reinterpret_cast<int *>(ws + L.rcv);
    int *d_err = reinterpret_cast<int *>(ws + L.err);
    const bool fused = L.state2 != L.coef;
    if (int rc = stage_positions3(g, src_x, src_y, src_z, rcv_x, rcv_y, rcv_z, d_src, d_rcv, st)) return rc;
    GB_CUDA(cudaMemsetAsync(d_err, 0, 4, st));
    GB_CUDA(cudaMemsetAsync(state, 0, (size_t)g.n_shots * 4 * g.vol * 4, st));
    if (fused) GB_CUDA(cudaMemsetAsync(state2, 0, (size_t)g.n_shots * 4 * g.vol * 4, st));
    GB_CUDA(cudaMemsetAsync(coef, 0, 6 * (size_t)g.vol * 4, st));
    float *eout[4] = {energy_p, energy_vx, energy_vy, energy_vz};
    const bool want_energy = energy_p && energy_vx && energy_vy && energy_vz;
    if ((energy_p || energy_vx || energy_vy || energy_vz) && !want_energy)
        return fail(GB_E_ARG, "give all four energy outputs or none");
    for (int f = 0; f < 4 && want_energy; ++f)
        GB_CUDA(cudaMemsetAsync(eout[f], 0, (size_t)g.nz * g.ny * g.nx * 4, st));

    Args3 A{};
    A.g = g;
    A.state = state;
    A.a1 = coef; A.k1 = coef + g.vol; A.a2 = coef + 2 * g.vol;
    A.k2 = coef + 3 * g.vol; A.k3 = coef + 4 * g.vol; A.k4 = coef + 5 * g.vol;
    A.src = d_src;
    A.wavelet = wavelet;
    for (int f = 0; f < 4; ++f) A.energy[f] = want_energy ? eout[f] : nullptr;
    coef3_kernel<<<4 * 148, 256, 0, st>>>(g, vp, rho, damp, desc->dz, coef, coef + g.vol, coef + 2 * g.vol,
                                          coef + 3 * g.vol, coef + 4 * g.vol, coef + 5 * g.vol);
    GB_CUDA(cudaGetLastError());
    const bool fs = desc->free_surface != 0;
    const bool want_tr = g.n_rcv > 0 && (trace_p || trace_vx || trace_vy || trace_vz);
    const size_t state_bytes = (size_t)g.n_shots * 4 * g.vol * 4;
    const size_t field = (size_t)g.n_shots * g.vol, blk = (imaging_rho ? 4 : 1) * field;
    Fused3 FU{};
    Fused3Args FA{};
    if (fused) {
        if (int rc = fused3_setup(g, state, state2, coef, want_energy, mode, &FU)) return rc;
        FA.free_surface = fs;
        FA.a2 = A.a2; FA.k2 = A.k2; FA.k3 = A.k3; FA.k4 = A.k4;
        FA.src = d_src;
        FA.wavelet = wavelet;
        for (int f = 0; f < 4; ++f) FA.energy[f] = A.energy[f];
        FA.err = d_err;
    }
    for (int it = 0; it < g.nt; ++it) {
        if (imaging) {   // this step's imaging fields, for a gradient without recompute
            A.img_i = FA.img_i = imaging + (size_t)it * blk;
            A.img_j = FA.img_j = imaging_rho ? A.img_i + field : nullptr;
        }
        const float *cur = fused ? FU.buf[FU.cur] : state;
        if (checkpoints && it % checkpoint_every == 0)   // the state before step it
            GB_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(checkpoints) + (size_t)(it / checkpoint_every) * state_bytes,
                                    cur, state_bytes, cudaMemcpyDeviceToDevice, st));
        if (fused) {
            if (int rc = fused3_step(g, FU, FA, it, st)) return rc;
        } else if (int rc = step3(g, A, it, fs, st)) {
            return rc;
        }
        if (want_tr)
            rec3_kernel<<<(g.n_shots * g.n_rcv + 255) / 256, 256, 0, st>>>(g, fused ? FU.buf[FU.cur] : state, d_rcv,
                                                                          trace_p, trace_vx, trace_vy, trace_vz, it,
                                                                          nullptr);
        GB_CUDA(cudaGetLastError());
    }
    return GB_OK;
}

namespace {

struct Layout3B {
    size_t err, state, state2, coef, src, rcv, lam_a, lam_b, img_i, img_j, g1, c1, g2, c2, total;
};

Layout3B layout3b(const Geo3 &g, int K, bool rho, int mode)
{
    Layout3B L{};
    size_t o = 0;
    const size_t st = (size_t)g.n_shots * 4 * g.vol * 4, f = (size_t)g.n_shots * g.vol * 4;
    L.err = o; o = align256(o + 4);
    L.state = o; o = align256(o + st);
    L.state2 = o; o = align256(o + (mode && K > 0 ? st : 0));
    L.coef = o; o = align256(o + 6 * (size_t)g.vol * 4);
    L.src = o; o = align256(o + 3 * (size_t)g.n_shots * 4);
    L.rcv = o; o = align256(o + 3 * (size_t)std::max(g.n_rcv, 1) * 4);
    L.lam_a = o; o = align256(o + st);
    L.lam_b = o; o = align256(o + st);
    L.img_i = o; o = align256(o + (size_t)K * f);
    L.img_j = o; o = align256(o + (rho ? 3 * (size_t)K * f : 0));
    L.g1 = o; o = align256(o + (size_t)g.vol * 4);
    L.c1 = o; o = align256(o + (size_t)g.vol * 4);
    L.g2 = o; o = align256(o + (rho ? (size_t)g.vol * 4 : 0));
    L.c2 = o; o = align256(o + (rho ? (size_t)g.vol * 4 : 0));
    L.total = o;
    return L;
}

}  // namespace

size_t gb3_imaging_bytes(const gb3_model_desc *desc, int32_t with_rho)
{
    Geo3 g;
    if (!geo3_of(desc, &g)) return 0;
    return (size_t)g.nt * (with_rho ? 4 : 1) * g.n_shots * g.vol * 4;
}

size_t gb3_backward_workspace_bytes(const gb3_model_desc *desc, int32_t checkpoint_every, int32_t with_rho)
{
    Geo3 g;
    if (!geo3_of(desc, &g) || checkpoint_every < 0) return 0;
    return layout3b(g, std::min<int>(checkpoint_every, g.nt), with_rho != 0, g_step3_fused.load()).total + 256;
}

int gb3_backward(const gb3_model_desc *desc, const int64_t *src_x, const int64_t *src_y, const int64_t *src_z,
                 const int64_t *rcv_x, const int64_t *rcv_y, const int64_t *rcv_z, const float *vp, const float *rho,
                 const float *damp, const float *wavelet, const float *res_p, const float *res_vx,
                 const float *res_vy, const float *res_vz, const float *checkpoints, int32_t checkpoint_every,
                 const float *imaging, int32_t imaging_rho, float *grad_vp, float *grad_rho, float *grad_wavelet,
                 void *workspace, size_t workspace_bytes, void *stream)
{
    gb::host::clear_error();
    Geo3 g;
    if (!geo3_of(desc, &g)) return fail(GB_E_ARG, "invalid 3-D model description");
    if (!vp || !rho || !damp || !wavelet || !grad_vp || (!checkpoints && !imaging))
        return fail(GB_E_ARG, "null argument");
    if (!imaging && checkpoint_every < 1) return fail(GB_E_ARG, "checkpoint_every must be >= 1");
    if (g.Nz > 65535) return fail(GB_E_ARG, "at most 65535 padded z planes");
    const bool with_rho = grad_rho != nullptr;
    if (imaging && with_rho && !imaging_rho)
        return fail(GB_E_ARG, "the density gradient needs imaging fields kept with imaging_rho");
    // with every step's imaging fields there is no recompute and no segment buffer
    const int K = imaging ? 0 : std::min<int>(checkpoint_every, g.nt);
    const int mode = g_step3_fused.load();
    const Layout3B L = layout3b(g, K, with_rho, mode);
    char *ws = aligned_ws(workspace);
    if (!workspace || workspace_bytes < L.total + (size_t)(ws - reinterpret_cast<char *>(workspace)))
        return fail(GB_E_WORKSPACE, "workspace too small");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    float *state = reinterpret_cast<float *>(ws + L.state);
    float *state2 = reinterpret_cast<float *>(ws + L.state2);
    const bool fused = L.state2 != L.coef;
    int *d_err = reinterpret_cast<int *>(ws + L.err);
    float *coef = reinterpret_cast<float *>(ws + L.coef);
    int *d_src = reinterpret_cast<int *>(ws + L.src), *d_rcv = reinterpret_cast<int *>(ws + L.rcv);
    float *lam_a = reinterpret_cast<float *>(ws + L.lam_a), *lam_b = reinterpret_cast<float *>(ws + L.lam_b);
    float *img_i = reinterpret_cast<float *>(ws + L.img_i), *img_j = reinterpret_cast<float *>(ws + L.img_j);
    float *G1 = reinterpret_cast<float *>(ws + L.g1), *C1 = reinterpret_cast<float *>(ws + L.c1);
    float *G2 = with_rho ? reinterpret_cast<float *>(ws + L.g2) : nullptr;
    float *C2 = with_rho ? reinterpret_cast<float *>(ws + L.c2) : nullptr;
    if (int rc = stage_positions3(g, src_x, src_y, src_z, rcv_x, rcv_y, rcv_z, d_src, d_rcv, st)) return rc;
    const size_t state_bytes = (size_t)g.n_shots * 4 * g.vol * 4, field = (size_t)g.n_shots * g.vol;
    GB_CUDA(cudaMemsetAsync(d_err, 0, 4, st));
    // columns [Nx, pitch) of both state buffers stay zero: a checkpoint brings them in as zeros
    if (fused) GB_CUDA(cudaMemsetAsync(state2, 0, state_bytes, st));
    GB_CUDA(cudaMemsetAsync(coef, 0, 6 * (size_t)g.vol * 4, st));
    GB_CUDA(cudaMemsetAsync(lam_a, 0, state_bytes, st));
    GB_CUDA(cudaMemsetAsync(lam_b, 0, state_bytes, st));
    GB_CUDA(cudaMemsetAsync(G1, 0, (size_t)g.vol * 4, st));
    GB_CUDA(cudaMemsetAsync(C1, 0, (size_t)g.vol * 4, st));
    if (with_rho) {
        GB_CUDA(cudaMemsetAsync(G2, 0, (size_t)g.vol * 4, st));
        GB_CUDA(cudaMemsetAsync(C2, 0, (size_t)g.vol * 4, st));
    }
    if (grad_wavelet) GB_CUDA(cudaMemsetAsync(grad_wavelet, 0, (size_t)g.n_shots * g.nt * 4, st));
    coef3_kernel<<<4 * 148, 256, 0, st>>>(g, vp, rho, damp, desc->dz, coef, coef + g.vol, coef + 2 * g.vol,
                                          coef + 3 * g.vol, coef + 4 * g.vol, coef + 5 * g.vol);
    GB_CUDA(cudaGetLastError());
    Args3 F{};
    F.g = g;
    F.state = state;
    F.a1 = coef; F.k1 = coef + g.vol; F.a2 = coef + 2 * g.vol;
    F.k2 = coef + 3 * g.vol; F.k3 = coef + 4 * g.vol; F.k4 = coef + 5 * g.vol;
    F.src = d_src;
    F.wavelet = wavelet;
    AdjArgs3 A{};
    A.g = g;
    A.a1 = F.a1; A.k1 = F.k1; A.a2 = F.a2; A.k2 = F.k2; A.k3 = F.k3; A.k4 = F.k4;
    A.G1 = G1; A.C1 = C1; A.G2 = G2; A.C2 = C2;
    const bool fs = desc->free_surface != 0;
    Fused3 FU{};
    Fused3Args FA{};
    if (fused) {
        if (int rc = fused3_setup(g, state, state2, coef, false, mode, &FU)) return rc;
        FA.free_surface = fs;
        FA.a2 = F.a2; FA.k2 = F.k2; FA.k3 = F.k3; FA.k4 = F.k4;
        FA.src = d_src;
        FA.wavelet = wavelet;
        FA.err = d_err;
    }
    const dim3 block(32, 4), grid((g.Nx + 127) / 128, (g.Ny + 3) / 4, g.Nz);
    const size_t blk = (imaging_rho ? 4 : 1) * field;      // one step of the caller's imaging buffer
    const int n_seg = imaging ? 1 : (g.nt + K - 1) / K;
    for (int seg = n_seg - 1; seg >= 0; --seg) {
        const int t0 = imaging ? 0 : seg * K, t1 = imaging ? g.nt : std::min(g.nt, t0 + K);
        if (!imaging) {
            // recompute the segment from its checkpoint, keeping the imaging fields
            GB_CUDA(cudaMemcpyAsync(state, reinterpret_cast<const char *>(checkpoints) + (size_t)seg * state_bytes,
                                    state_bytes, cudaMemcpyDeviceToDevice, st));
            FU.cur = 0;   // FU.buf[0] is `state`
            for (int it = t0; it < t1; ++it) {
                F.img_i = FA.img_i = img_i + (size_t)(it - t0) * field;
                F.img_j = FA.img_j = with_rho ? img_j + (size_t)(it - t0) * 3 * field : nullptr;
                if (fused) {
                    if (int rc = fused3_step(g, FU, FA, it, st)) return rc;
                } else if (int rc = step3(g, F, it, fs, st)) {
                    return rc;
                }
            }
        }
        // adjoint steps, last to first
        for (int it = t1 - 1; it >= t0; --it) {
            if (g.n_rcv > 0 && (res_p || res_vx || res_vy || res_vz))
                inj3_kernel<<<(g.n_shots * g.n_rcv + 255) / 256, 256, 0, st>>>(g, lam_a, d_rcv, res_p, res_vx,
                                                                              res_vy, res_vz, it);
            if (fs) fold3_kernel<<<148, 256, 0, st>>>(g, lam_a, 3, 1, 1.f);
            if (imaging) {
                A.img_i = imaging + (size_t)it * blk;
                A.img_j = with_rho ? imaging + (size_t)it * blk + field : nullptr;
            } else {
                A.img_i = img_i + (size_t)(it - t0) * field;
                A.img_j = with_rho ? img_j + (size_t)(it - t0) * 3 * field : nullptr;
            }
            A.lam_in = lam_a;
            A.lam_out = lam_b;
            adj_v3_kernel<<<grid, block, 0, st>>>(A);
            if (fs) fold3_kernel<<<148, 256, 0, st>>>(g, lam_b, 0, 2, -1.f);
            if (grad_wavelet)
                wavelet_grad3_kernel<<<(g.n_shots + 127) / 128, 128, 0, st>>>(g, lam_b, d_src, grad_wavelet, it);
            A.lam_in = lam_b;
            A.lam_out = lam_a;
            adj_p3_kernel<<<grid, block, 0, st>>>(A);
            GB_CUDA(cudaGetLastError());
        }
    }
    grad3_finish_kernel<<<4 * 148, 256, 0, st>>>(g, vp, rho, desc->dz, G1, C1, G2, C2, grad_vp, grad_rho);
    GB_CUDA(cudaGetLastError());
    return GB_OK;
}

}  // extern "C"
