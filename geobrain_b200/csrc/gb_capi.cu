// C ABI of the B200 acoustic propagator (declared in include/geobrain_b200.h):
// plans, workspace layout, TMA descriptors and the host-side time loops.
#include "../../include/geobrain_b200.h"

#include "gb_adj.cuh"
#include "gb_aux.cuh"
#include "gb_fwd.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using namespace gb;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

#define GB_CUDA(call)                                                                        \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(GB_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

// ---------------------------------------------------------------------------
// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

int get_encoder(PFN_cuTensorMapEncodeTiled_v12000 *out)
{
    std::call_once(g_encode_once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!g_encode) return fail(GB_E_CUDA, "cuTensorMapEncodeTiled unavailable");
    *out = g_encode;
    return GB_OK;
}

// 3-D map over a field buffer laid out [n_planes][Nz][pitch] fp32, valid
// extent Nx columns (columns >= Nx and rows outside [0, Nz) read as zero).
int make_map(CUtensorMap *map, const float *base, int Nx, int Nz, int pitch, int n_planes, int box_x,
             int box_z)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc;
    if (int rc = get_encoder(&enc)) return rc;
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (pitch % 4))
        return fail(GB_E_ARG, "field buffer not 16-byte aligned");
    cuuint64_t dims[3] = {(cuuint64_t)Nx, (cuuint64_t)Nz, (cuuint64_t)n_planes};
    cuuint64_t strides[2] = {(cuuint64_t)pitch * 4, (cuuint64_t)pitch * 4 * Nz};
    cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_z, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(GB_E_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return GB_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------
struct gb_plan {
    gb_model_desc d{};
    int R = 2, fs = 1;
    int Nz = 0, Nx = 0, pitch = 0;
    long long plane = 0;
    int tz = 32, spc = 0;   // tile rows, shots per CTA
    int tiles_x = 0, tiles_z = 0, n_tiles = 0, n_groups = 0;
    float c[4] = {0, 0, 0, 0};
    std::vector<int> src_z, src_x, rcv_z, rcv_x;   // padded
    std::vector<int> rcv_ptr;                      // CSR over tiles (own receivers)
    std::vector<int4> rcv_ent;
    std::vector<int> arcv_ptr;                     // CSR over tiles: receivers inside the
    std::vector<int4> arcv_ent;                    // loaded halo rectangles (adjoint)
    // optional phase profiling: event pairs recorded on the launching stream
    bool prof = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[3];   // forward, recompute, adjoint
    long long launches = 0;

    ~gb_plan() { clear_events(); }
    void clear_events()
    {
        for (auto &v : ev) {
            for (auto &e : v) {
                cudaEventDestroy(e.first);
                cudaEventDestroy(e.second);
            }
            v.clear();
        }
    }
    // record the start (end) of a phase; returns the index of the pair
    void mark(int phase, bool start, cudaStream_t st)
    {
        if (!prof) return;
        if (start) {
            cudaEvent_t a, b;
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            ev[phase].push_back({a, b});
            cudaEventRecord(a, st);
        } else if (!ev[phase].empty()) {
            cudaEventRecord(ev[phase].back().second, st);
        }
    }

    void retile()
    {
        tiles_x = (Nx + TX - 1) / TX;
        tiles_z = (Nz + tz - 1) / tz;
        n_tiles = tiles_x * tiles_z;
        if (spc <= 0) spc = default_spc();
        n_groups = (d.n_shots + spc - 1) / spc;
        rcv_ptr.assign(n_tiles + 1, 0);
        for (int r = 0; r < d.n_rcv; ++r) rcv_ptr[(rcv_z[r] / tz) * tiles_x + rcv_x[r] / TX + 1]++;
        for (int t = 0; t < n_tiles; ++t) rcv_ptr[t + 1] += rcv_ptr[t];
        rcv_ent.assign(d.n_rcv, int4{0, 0, 0, 0});
        std::vector<int> fill(rcv_ptr.begin(), rcv_ptr.end() - 1);
        for (int r = 0; r < d.n_rcv; ++r) {
            const int t = (rcv_z[r] / tz) * tiles_x + rcv_x[r] / TX;
            rcv_ent[fill[t]++] = int4{rcv_z[r] - (rcv_z[r] / tz) * tz, rcv_x[r] - (rcv_x[r] / TX) * TX, r, 0};
        }
        // adjoint: every tile whose halo rectangles [z0-2R, z0+tz+2R) x
        // [x0-8, x0+TX+8) contain the receiver injects it into its copy
        arcv_ptr.assign(n_tiles + 1, 0);
        arcv_ent.clear();
        std::vector<std::vector<int4>> per(n_tiles);
        for (int r = 0; r < d.n_rcv; ++r) {
            const int z = rcv_z[r], x = rcv_x[r];
            // candidate tiles (a superset; the test below is exact)
            const int tz_lo = std::max(0, (z - 2 * R) / tz - 1), tz_hi = std::min(tiles_z - 1, (z + 2 * R) / tz + 1);
            const int tx_lo = std::max(0, (x - 8) / TX - 1), tx_hi = std::min(tiles_x - 1, (x + 8) / TX + 1);
            for (int a = tz_lo; a <= tz_hi; ++a)
                for (int b = tx_lo; b <= tx_hi; ++b) {
                    const int z0 = a * tz, x0 = b * TX;
                    if (z >= z0 - 2 * R && z < z0 + tz + 2 * R && x >= x0 - 8 && x < x0 + TX + 8)
                        per[a * tiles_x + b].push_back(int4{z, x, r, 0});
                }
        }
        for (int t = 0; t < n_tiles; ++t) {
            arcv_ptr[t + 1] = arcv_ptr[t] + (int)per[t].size();
            arcv_ent.insert(arcv_ent.end(), per[t].begin(), per[t].end());
        }
    }

    // Enough CTAs to fill the GPU several times over, as few groups as that
    // allows (each group re-reads the coefficient tiles and adds its own
    // energy partial sums).
    int default_spc() const
    {
        const int S = d.n_shots;
        int best = S;
        for (int spc_try = S; spc_try >= 1; --spc_try) {
            const long long ctas = (long long)n_tiles * ((S + spc_try - 1) / spc_try);
            best = spc_try;
            if (ctas >= 4 * 148) break;
        }
        return std::max(1, std::min(best, 8));
    }

    StepGeom geom() const
    {
        StepGeom g{};
        g.Nz = Nz; g.Nx = Nx; g.pitch = pitch;
        g.nz = d.nz; g.nx = d.nx; g.pml = d.nabc; g.fs = fs;
        g.p_r0 = std::max(fs + 1, R); g.p_r1 = Nz - 1 - R; g.p_c0 = R; g.p_c1 = Nx - 1 - R;
        g.vx_r0 = fs; g.vx_r1 = Nz - 2; g.vx_c0 = R - 1; g.vx_c1 = Nx - 1 - R;
        g.vz_r0 = std::max(fs, R - 1); g.vz_r1 = Nz - 1 - R; g.vz_c0 = 1; g.vz_c1 = Nx - 2;
        g.tiles_x = tiles_x; g.n_tiles = n_tiles;
        g.n_shots = d.n_shots; g.shots_per_cta = spc; g.n_groups = n_groups;
        g.nt = d.nt; g.n_rcv = d.n_rcv;
        g.dt = d.dt;
        for (int k = 0; k < 4; ++k) g.c[k] = c[k];
        g.plane = plane;
        return g;
    }
};

namespace {

// Workspace layout (offsets in bytes from the 256-aligned base).
struct Layout {
    size_t err, coef, fields, energy, src, rcv_ptr, rcv_ent, total;
    // gradient only
    size_t mu, img, g1, c1, g2, c2, arcv_ptr, arcv_ent;
    int n_img;
};

// with_gradient: 0 forward only, 1 velocity gradient, 2 velocity and density.
Layout layout(const gb_plan *p, int with_gradient = 0, int checkpoint_every = 0)
{
    Layout L{};
    size_t o = 0;
    const size_t S = p->d.n_shots;
    L.err = o; o += 256;
    L.coef = o; o = align256(o + 5 * p->plane * 4);
    L.fields = o; o = align256(o + 2 * S * 3 * p->plane * 4);
    L.energy = o; o = align256(o + 3 * p->plane * 4);
    L.src = o; o = align256(o + 2 * S * 4);
    L.rcv_ptr = o; o = align256(o + (p->n_tiles + 1) * 4);
    L.rcv_ent = o; o = align256(o + std::max<size_t>(p->d.n_rcv, 1) * 16);
    L.n_img = with_gradient >= 2 ? 3 : 1;
    if (with_gradient > 0) {
        const size_t K = std::max(1, std::min(checkpoint_every, p->d.nt));
        const size_t G = p->n_groups;
        L.mu = o; o = align256(o + 2 * S * 3 * p->plane * 4);
        L.img = o; o = align256(o + K * L.n_img * S * p->plane * 4);
        L.g1 = o; o = align256(o + G * p->plane * 4);
        L.c1 = o; o = align256(o + G * p->plane * 4);
        if (with_gradient >= 2) {
            L.g2 = o; o = align256(o + G * p->plane * 4);
            L.c2 = o; o = align256(o + G * p->plane * 4);
        }
        L.arcv_ptr = o; o = align256(o + (p->n_tiles + 1) * 4);
        L.arcv_ent = o; o = align256(o + std::max<size_t>(p->arcv_ent.size(), 1) * 16);
    }
    L.total = o;
    return L;
}

template <int R, int TZ, bool FS, bool EN, int IMG>
void *fwd_fn()
{
    return reinterpret_cast<void *>(&fwd_step_kernel<R, TZ, FS, EN, IMG>);
}

// Energy sums are only taken by the plain forward; the imaging fields only by
// the gradient's recompute (which takes no energy).
template <int R, int TZ>
void *fwd_pick3(bool fs, bool en, int img)
{
    if (fs) {
        if (img == 1) return fwd_fn<R, TZ, true, false, 1>();
        if (img == 2) return fwd_fn<R, TZ, true, false, 2>();
        return en ? fwd_fn<R, TZ, true, true, 0>() : fwd_fn<R, TZ, true, false, 0>();
    }
    if (img == 1) return fwd_fn<R, TZ, false, false, 1>();
    if (img == 2) return fwd_fn<R, TZ, false, false, 2>();
    return en ? fwd_fn<R, TZ, false, true, 0>() : fwd_fn<R, TZ, false, false, 0>();
}

struct FwdKernel {
    void *fn;
    size_t smem;
};

FwdKernel fwd_kernel(int R, int tz, bool fs, bool en, int im)
{
    FwdKernel k{nullptr, 0};
    if (R == 2 && tz == 32) { k.fn = fwd_pick3<2, 32>(fs, en, im); k.smem = en ? fwd_smem_bytes<2, 32, true>() : fwd_smem_bytes<2, 32, false>(); }
    if (R == 2 && tz == 16) { k.fn = fwd_pick3<2, 16>(fs, en, im); k.smem = en ? fwd_smem_bytes<2, 16, true>() : fwd_smem_bytes<2, 16, false>(); }
    if (R == 4 && tz == 32) { k.fn = fwd_pick3<4, 32>(fs, en, im); k.smem = en ? fwd_smem_bytes<4, 32, true>() : fwd_smem_bytes<4, 32, false>(); }
    if (R == 4 && tz == 16) { k.fn = fwd_pick3<4, 16>(fs, en, im); k.smem = en ? fwd_smem_bytes<4, 16, true>() : fwd_smem_bytes<4, 16, false>(); }
    return k;
}

template <int R, int TZ>
void *adj_pick(bool fs, bool rho)
{
    if (fs) return rho ? reinterpret_cast<void *>(&adj_step_kernel<R, TZ, true, true>)
                       : reinterpret_cast<void *>(&adj_step_kernel<R, TZ, true, false>);
    return rho ? reinterpret_cast<void *>(&adj_step_kernel<R, TZ, false, true>)
               : reinterpret_cast<void *>(&adj_step_kernel<R, TZ, false, false>);
}

FwdKernel adj_kernel(int R, int tz, bool fs, bool rho)
{
    FwdKernel k{nullptr, 0};
    if (R == 2 && tz == 32) { k.fn = adj_pick<2, 32>(fs, rho); k.smem = adj_smem_bytes<2, 32>(); }
    if (R == 2 && tz == 16) { k.fn = adj_pick<2, 16>(fs, rho); k.smem = adj_smem_bytes<2, 16>(); }
    if (R == 4 && tz == 32) { k.fn = adj_pick<4, 32>(fs, rho); k.smem = adj_smem_bytes<4, 32>(); }
    if (R == 4 && tz == 16) { k.fn = adj_pick<4, 16>(fs, rho); k.smem = adj_smem_bytes<4, 16>(); }
    return k;
}

int box_rows_p(int R, int tz) { return tz + 2 * R; }
int box_rows_vz(int R, int tz) { return tz + 4 * R; }

struct Maps {
    CUtensorMap p, vx, vz;
};

int make_maps(const gb_plan *P, const float *buf, Maps *m)
{
    const int n_planes = 3 * P->d.n_shots;
    if (int rc = make_map(&m->p, buf, P->Nx, P->Nz, P->pitch, n_planes, RW, box_rows_p(P->R, P->tz))) return rc;
    if (int rc = make_map(&m->vx, buf, P->Nx, P->Nz, P->pitch, n_planes, VXW, box_rows_p(P->R, P->tz))) return rc;
    return make_map(&m->vz, buf, P->Nx, P->Nz, P->pitch, n_planes, RW, box_rows_vz(P->R, P->tz));
}

template <class Args>
int launch_step(gb_plan *P, const FwdKernel &K, const Maps &maps, const Args &A, cudaStream_t st)
{
    void *args[] = {(void *)&maps.p, (void *)&maps.vx, (void *)&maps.vz, (void *)&A};
    dim3 grid(P->n_tiles * P->n_groups), block(NTHR);
    GB_CUDA(cudaLaunchKernel(K.fn, grid, block, args, K.smem, st));
    ++P->launches;
    return GB_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char *gb_last_error(void) { return g_last_error.c_str(); }

const char *gb_version(void) { return "geobrain_b200 0.1 (sm_100a)"; }

int gb_plan_create(const gb_model_desc *desc, const int64_t *src_x, const int64_t *src_z, const int64_t *rcv_x,
                   const int64_t *rcv_z, gb_plan **out)
{
    g_last_error.clear();
    if (!desc || !out) return fail(GB_E_ARG, "null argument");
    *out = nullptr;
    const gb_model_desc &d = *desc;
    if (d.half != 2 && d.half != 4) return fail(GB_E_ARG, "half must be 2 (4th order) or 4 (8th order)");
    if (d.nz < 1 || d.nx < 1 || d.nt < 1 || d.n_shots < 1 || d.n_rcv < 0)
        return fail(GB_E_ARG, "sizes must be positive");
    if (d.nabc < d.half) return fail(GB_E_ARG, "nabc must be at least the stencil half-width");
    if (!(d.dt > 0.f) || !(d.dx > 0.f)) return fail(GB_E_ARG, "dt and dx must be positive");
    if (d.n_shots > 65535) return fail(GB_E_ARG, "too many shots");
    const long long Nz = (long long)d.nz + 2 * d.nabc, Nx = (long long)d.nx + 2 * d.nabc;
    if (Nz > (1 << 20) || Nx > (1 << 20)) return fail(GB_E_ARG, "grid too large");
    if ((d.n_shots && (!src_x || !src_z)) || (d.n_rcv && (!rcv_x || !rcv_z)))
        return fail(GB_E_ARG, "null position array");
    gb_plan *p = new gb_plan();
    p->d = d;
    p->R = d.half;
    p->fs = d.free_surface ? d.nabc : 1;
    p->Nz = (int)Nz;
    p->Nx = (int)Nx;
    p->pitch = (int)((Nx + 31) / 32 * 32);
    p->plane = (long long)p->Nz * p->pitch;
    if (d.half == 2) {
        p->c[0] = 9.0f / 8.0f;
        p->c[1] = (float)(-1.0 / 24.0);
    } else {
        // staggered Taylor coefficients of half-width 4 (fd_coefficients(4, 's'))
        p->c[0] = (float)(1225.0 / 1024.0);
        p->c[1] = (float)(-245.0 / 3072.0);
        p->c[2] = (float)(49.0 / 5120.0);
        p->c[3] = (float)(-5.0 / 7168.0);
    }
    for (int s = 0; s < d.n_shots; ++s) {
        const long long z = src_z[s] + d.nabc, x = src_x[s] + d.nabc;
        if (z < 0 || z >= Nz || x < 0 || x >= Nx) {
            delete p;
            return fail(GB_E_ARG, "source " + std::to_string(s) + " outside the padded grid");
        }
        p->src_z.push_back((int)z);
        p->src_x.push_back((int)x);
    }
    for (int r = 0; r < d.n_rcv; ++r) {
        const long long z = rcv_z[r] + d.nabc, x = rcv_x[r] + d.nabc;
        // vx is (Nz, Nx-1) and vz (Nz-1, Nx) in the reference: a receiver must
        // index all three fields.
        if (z < 0 || z >= Nz - 1 || x < 0 || x >= Nx - 1) {
            delete p;
            return fail(GB_E_ARG, "receiver " + std::to_string(r) + " outside the padded grid");
        }
        p->rcv_z.push_back((int)z);
        p->rcv_x.push_back((int)x);
    }
    p->retile();
    *out = p;
    return GB_OK;
}

void gb_plan_destroy(gb_plan *plan) { delete plan; }

int gb_plan_set_tiling(gb_plan *p, int tile_rows, int shots_per_cta)
{
    if (!p) return fail(GB_E_ARG, "null plan");
    if (tile_rows != 0 && tile_rows != 16 && tile_rows != 32) return fail(GB_E_ARG, "tile_rows must be 16 or 32");
    if (shots_per_cta < 0) return fail(GB_E_ARG, "shots_per_cta must be >= 0");
    if (tile_rows) p->tz = tile_rows;
    p->spc = shots_per_cta ? std::min(shots_per_cta, p->d.n_shots) : 0;
    p->retile();
    return GB_OK;
}

size_t gb_plan_workspace_bytes(const gb_plan *p, int with_gradient, int checkpoint_every)
{
    if (!p) return 0;
    return layout(p, with_gradient, checkpoint_every).total + 256;
}

size_t gb_plan_checkpoint_bytes(const gb_plan *p, int checkpoint_every, int ckpt_format)
{
    if (!p || checkpoint_every < 1) return 0;
    const size_t n_ck = (p->d.nt + checkpoint_every - 1) / checkpoint_every;
    const size_t per = (size_t)p->d.n_shots * 3 * p->plane;
    if (ckpt_format == GB_CKPT_F32) return n_ck * per * 4;
    return n_ck * (align256(per * 2) + align256((size_t)p->d.n_shots * 3 * 4));
}

int gb_forward(gb_plan *P, const float *vp, const float *rho, const float *damp, const float *wavelet,
               float *trace_p, float *trace_vx, float *trace_vz, float *energy_p, float *energy_vx,
               float *energy_vz, int32_t snapshot_every, float *snapshots, void *checkpoints,
               int32_t checkpoint_every, int32_t ckpt_format, void *workspace, size_t workspace_bytes,
               void *stream)
{
    g_last_error.clear();
    if (!P || !vp || !rho || !damp || !wavelet) return fail(GB_E_ARG, "null argument");
    if (checkpoints && ckpt_format != GB_CKPT_F32) return fail(GB_E_UNSUPPORTED, "checkpoint format not built yet");
    const Layout L = layout(P);
    char *ws = reinterpret_cast<char *>(align256(reinterpret_cast<uintptr_t>(workspace)));
    if (!workspace || workspace_bytes < L.total + (size_t)(ws - reinterpret_cast<char *>(workspace)))
        return fail(GB_E_WORKSPACE, "workspace too small");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const gb_model_desc &d = P->d;
    const int S = d.n_shots;
    const bool want_energy = energy_p || energy_vx || energy_vz;

    int *err = reinterpret_cast<int *>(ws + L.err);
    float *coef = reinterpret_cast<float *>(ws + L.coef);
    float *a1 = coef, *k1 = coef + P->plane, *a2 = coef + 2 * P->plane, *k2 = coef + 3 * P->plane,
          *k3 = coef + 4 * P->plane;
    float *buf[2] = {reinterpret_cast<float *>(ws + L.fields),
                     reinterpret_cast<float *>(ws + L.fields) + (size_t)S * 3 * P->plane};
    float *energy = reinterpret_cast<float *>(ws + L.energy);
    int *d_src = reinterpret_cast<int *>(ws + L.src);
    int *d_rptr = reinterpret_cast<int *>(ws + L.rcv_ptr);
    int4 *d_rent = reinterpret_cast<int4 *>(ws + L.rcv_ent);

    GB_CUDA(cudaMemsetAsync(err, 0, 4, st));
    GB_CUDA(cudaMemcpyAsync(d_src, P->src_z.data(), S * 4, cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemcpyAsync(d_src + S, P->src_x.data(), S * 4, cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemcpyAsync(d_rptr, P->rcv_ptr.data(), (P->n_tiles + 1) * 4, cudaMemcpyHostToDevice, st));
    if (d.n_rcv)
        GB_CUDA(cudaMemcpyAsync(d_rent, P->rcv_ent.data(), d.n_rcv * 16, cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemsetAsync(buf[0], 0, (size_t)S * 3 * P->plane * 4, st));
    GB_CUDA(cudaMemsetAsync(buf[1], 0, (size_t)S * 3 * P->plane * 4, st));
    if (want_energy) GB_CUDA(cudaMemsetAsync(energy, 0, 3 * P->plane * 4, st));

    P->mark(0, true, st);
    coef_kernel<<<4 * 148, 256, 0, st>>>(vp, rho, damp, d.nz, d.nx, d.nabc, P->Nz, P->Nx, P->pitch, P->fs, d.dt,
                                         d.dx, a1, k1, a2, k2, k3);
    GB_CUDA(cudaGetLastError());
    ++P->launches;

    FwdKernel K = fwd_kernel(P->R, P->tz, d.free_surface != 0, want_energy, 0);
    if (!K.fn) return fail(GB_E_UNSUPPORTED, "no kernel for this configuration");
    GB_CUDA(cudaFuncSetAttribute(K.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K.smem));
    Maps maps[2];
    for (int b = 0; b < 2; ++b)
        if (int rc = make_maps(P, buf[b], &maps[b])) return rc;

    FwdArgs A{};
    A.g = P->geom();
    A.a1 = a1; A.k1 = k1; A.a2 = a2; A.k2 = k2; A.k3 = k3;
    A.src_z = d_src; A.src_x = d_src + S;
    A.wavelet = wavelet;
    A.rcv_ptr = d_rptr; A.rcv_ent = d_rent;
    A.tr_p = trace_p; A.tr_vx = trace_vx; A.tr_vz = trace_vz;
    A.energy = want_energy ? energy : nullptr;
    A.imaging = nullptr;
    A.err = err;

    const size_t state_bytes = (size_t)S * 3 * P->plane * 4;
    int snap_i = 0;
    for (int it = 0; it < d.nt; ++it) {
        const int b = it & 1;
        if (checkpoints && checkpoint_every > 0 && it % checkpoint_every == 0)
            GB_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(checkpoints) + (size_t)(it / checkpoint_every) * state_bytes,
                                    buf[b], state_bytes, cudaMemcpyDeviceToDevice, st));
        A.it = it;
        A.out = buf[b ^ 1];
        if (int rc = launch_step(P, K, maps[b], A, st)) return rc;
        if (snapshot_every > 0 && snapshots && ((it + 1) % snapshot_every == 0 || it == d.nt - 1)) {
            GB_CUDA(cudaMemcpy2DAsync(snapshots + (size_t)snap_i * d.nz * d.nx, (size_t)d.nx * 4,
                                      buf[b ^ 1] + (size_t)d.nabc * P->pitch + d.nabc, (size_t)P->pitch * 4,
                                      (size_t)d.nx * 4, d.nz, cudaMemcpyDeviceToDevice, st));
            ++snap_i;
        }
    }
    float *eouts[3] = {energy_p, energy_vx, energy_vz};
    for (int f = 0; f < 3; ++f)
        if (eouts[f]) {
            extract_interior_kernel<<<148, 256, 0, st>>>(energy + f * P->plane, d.nz, d.nx, d.nabc, P->pitch,
                                                         eouts[f]);
            GB_CUDA(cudaGetLastError());
            ++P->launches;
        }
    P->mark(0, false, st);
    return GB_OK;
}

int gb_backward(gb_plan *P, const float *vp, const float *rho, const float *damp, const float *wavelet,
                const float *res_p, const float *res_vx, const float *res_vz, const void *checkpoints,
                int32_t checkpoint_every, int32_t ckpt_format, float *grad_vp, float *grad_rho, void *workspace,
                size_t workspace_bytes, void *stream)
{
    g_last_error.clear();
    if (!P || !vp || !rho || !damp || !wavelet || !checkpoints || !grad_vp) return fail(GB_E_ARG, "null argument");
    if (checkpoint_every < 1) return fail(GB_E_ARG, "checkpoint_every must be >= 1");
    if (ckpt_format != GB_CKPT_F32) return fail(GB_E_UNSUPPORTED, "checkpoint format not built yet");
    const gb_model_desc &d = P->d;
    const int S = d.n_shots;
    const int K = std::min<int>(checkpoint_every, d.nt);
    const int with_grad = grad_rho ? 2 : 1;
    const Layout L = layout(P, with_grad, K);
    char *ws = reinterpret_cast<char *>(align256(reinterpret_cast<uintptr_t>(workspace)));
    if (!workspace || workspace_bytes < L.total + (size_t)(ws - reinterpret_cast<char *>(workspace)))
        return fail(GB_E_WORKSPACE, "workspace too small");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

    int *err = reinterpret_cast<int *>(ws + L.err);
    float *coef = reinterpret_cast<float *>(ws + L.coef);
    float *a1 = coef, *k1 = coef + P->plane, *a2 = coef + 2 * P->plane, *k2 = coef + 3 * P->plane,
          *k3 = coef + 4 * P->plane;
    const size_t state_fl = (size_t)S * 3 * P->plane;
    float *fb[2] = {reinterpret_cast<float *>(ws + L.fields), reinterpret_cast<float *>(ws + L.fields) + state_fl};
    float *mu[2] = {reinterpret_cast<float *>(ws + L.mu), reinterpret_cast<float *>(ws + L.mu) + state_fl};
    float *img = reinterpret_cast<float *>(ws + L.img);
    float *G1 = reinterpret_cast<float *>(ws + L.g1), *C1 = reinterpret_cast<float *>(ws + L.c1);
    float *G2 = with_grad >= 2 ? reinterpret_cast<float *>(ws + L.g2) : nullptr;
    float *C2 = with_grad >= 2 ? reinterpret_cast<float *>(ws + L.c2) : nullptr;
    int *d_src = reinterpret_cast<int *>(ws + L.src);
    int *d_rptr = reinterpret_cast<int *>(ws + L.rcv_ptr);
    int4 *d_rent = reinterpret_cast<int4 *>(ws + L.rcv_ent);
    int *d_aptr = reinterpret_cast<int *>(ws + L.arcv_ptr);
    int4 *d_aent = reinterpret_cast<int4 *>(ws + L.arcv_ent);

    GB_CUDA(cudaMemsetAsync(err, 0, 4, st));
    GB_CUDA(cudaMemcpyAsync(d_src, P->src_z.data(), S * 4, cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemcpyAsync(d_src + S, P->src_x.data(), S * 4, cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemcpyAsync(d_rptr, P->rcv_ptr.data(), (P->n_tiles + 1) * 4, cudaMemcpyHostToDevice, st));
    if (d.n_rcv) GB_CUDA(cudaMemcpyAsync(d_rent, P->rcv_ent.data(), d.n_rcv * 16, cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemcpyAsync(d_aptr, P->arcv_ptr.data(), (P->n_tiles + 1) * 4, cudaMemcpyHostToDevice, st));
    if (!P->arcv_ent.empty())
        GB_CUDA(cudaMemcpyAsync(d_aent, P->arcv_ent.data(), P->arcv_ent.size() * 16, cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemsetAsync(mu[0], 0, 2 * state_fl * 4, st));
    GB_CUDA(cudaMemsetAsync(G1, 0, (size_t)P->n_groups * P->plane * 4, st));
    GB_CUDA(cudaMemsetAsync(C1, 0, (size_t)P->n_groups * P->plane * 4, st));
    if (G2) {
        GB_CUDA(cudaMemsetAsync(G2, 0, (size_t)P->n_groups * P->plane * 4, st));
        GB_CUDA(cudaMemsetAsync(C2, 0, (size_t)P->n_groups * P->plane * 4, st));
    }
    coef_kernel<<<4 * 148, 256, 0, st>>>(vp, rho, damp, d.nz, d.nx, d.nabc, P->Nz, P->Nx, P->pitch, P->fs, d.dt,
                                         d.dx, a1, k1, a2, k2, k3);
    GB_CUDA(cudaGetLastError());
    ++P->launches;

    const bool fs = d.free_surface != 0;
    FwdKernel KF = fwd_kernel(P->R, P->tz, fs, false, with_grad);
    FwdKernel KA = adj_kernel(P->R, P->tz, fs, with_grad >= 2);
    if (!KF.fn || !KA.fn) return fail(GB_E_UNSUPPORTED, "no kernel for this configuration");
    GB_CUDA(cudaFuncSetAttribute(KF.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KF.smem));
    GB_CUDA(cudaFuncSetAttribute(KA.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KA.smem));
    Maps fmaps[2], amaps[2];
    for (int b = 0; b < 2; ++b) {
        if (int rc = make_maps(P, fb[b], &fmaps[b])) return rc;
        if (int rc = make_maps(P, mu[b], &amaps[b])) return rc;
    }

    const StepGeom g = P->geom();
    FwdArgs F{};
    F.g = g;
    F.a1 = a1; F.k1 = k1; F.a2 = a2; F.k2 = k2; F.k3 = k3;
    F.src_z = d_src; F.src_x = d_src + S;
    F.wavelet = wavelet;
    F.rcv_ptr = d_rptr; F.rcv_ent = d_rent;
    F.err = err;
    F.img_field_stride = (long long)S * P->plane;
    AdjArgs A{};
    A.g = g;
    A.a1 = a1; A.k1 = k1; A.a2 = a2; A.k2 = k2; A.k3 = k3;
    A.rcv_ptr = d_aptr; A.rcv_ent = d_aent;
    A.res_p = res_p; A.res_vx = res_vx; A.res_vz = res_vz;
    A.img_field_stride = (long long)S * P->plane;
    A.G1 = G1; A.C1 = C1; A.G2 = G2; A.C2 = C2;
    A.err = err;

    const size_t step_img = (size_t)L.n_img * S * P->plane;
    const int n_seg = (d.nt + K - 1) / K;
    int cur = 0;
    for (int seg = n_seg - 1; seg >= 0; --seg) {
        const int t0 = seg * K, t1 = std::min(d.nt, t0 + K);
        GB_CUDA(cudaMemcpyAsync(fb[0], reinterpret_cast<const char *>(checkpoints) + (size_t)seg * state_fl * 4,
                                state_fl * 4, cudaMemcpyDeviceToDevice, st));
        P->mark(1, true, st);
        for (int it = t0; it < t1; ++it) {
            const int b = (it - t0) & 1;
            F.it = it;
            F.out = fb[b ^ 1];
            F.imaging = img + (size_t)(it - t0) * step_img;
            if (int rc = launch_step(P, KF, fmaps[b], F, st)) return rc;
        }
        P->mark(1, false, st);
        P->mark(2, true, st);
        for (int it = t1 - 1; it >= t0; --it) {
            A.it = it;
            A.out = mu[cur ^ 1];
            A.img = img + (size_t)(it - t0) * step_img;
            if (int rc = launch_step(P, KA, amaps[cur], A, st)) return rc;
            cur ^= 1;
        }
        P->mark(2, false, st);
    }
    grad_finish_kernel<<<4 * 148, 256, 0, st>>>(vp, rho, G1, C1, G2, C2, P->n_groups, P->plane, d.nz, d.nx, d.nabc,
                                                P->pitch, grad_vp, grad_rho);
    GB_CUDA(cudaGetLastError());
    ++P->launches;
    return GB_OK;
}

int gb_plan_set_profiling(gb_plan *P, int enable)
{
    if (!P) return fail(GB_E_ARG, "null plan");
    P->prof = enable != 0;
    P->clear_events();
    P->launches = 0;
    return GB_OK;
}

int gb_plan_profile(gb_plan *P, double *ms_forward, double *ms_recompute, double *ms_adjoint, long long *launches)
{
    if (!P) return fail(GB_E_ARG, "null plan");
    double *outs[3] = {ms_forward, ms_recompute, ms_adjoint};
    for (int ph = 0; ph < 3; ++ph) {
        double sum = 0.0;
        for (auto &e : P->ev[ph]) {
            float ms = 0.f;
            GB_CUDA(cudaEventSynchronize(e.second));
            GB_CUDA(cudaEventElapsedTime(&ms, e.first, e.second));
            sum += ms;
        }
        if (outs[ph]) *outs[ph] = sum;
    }
    if (launches) *launches = P->launches;
    P->clear_events();
    P->launches = 0;
    return GB_OK;
}

int gb_workspace_status(const void *workspace, void *stream)
{
    g_last_error.clear();
    if (!workspace) return fail(GB_E_ARG, "null workspace");
    const char *ws = reinterpret_cast<const char *>(align256(reinterpret_cast<uintptr_t>(workspace)));
    int flag = 0;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    GB_CUDA(cudaMemcpyAsync(&flag, ws, 4, cudaMemcpyDeviceToHost, st));
    GB_CUDA(cudaStreamSynchronize(st));
    if (flag == GB_E_TIMEOUT) return fail(GB_E_TIMEOUT, "a device-side wait timed out");
    if (flag != 0) return fail(flag, "device error flag set");
    return GB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Forward modelling for callers that cannot allocate device memory.
//
// Some hosts cannot call cudaMalloc or hand the library a workspace: plugins
// embedded in an application whose memory pool owns all device memory and
// exposes no allocation hook, or code paths where the caller's allocator must
// not be re-entered.  For them the scratch gb_forward needs (coefficient
// planes, the two time levels of the wavefield, the energy sums and the
// receiver tables) lives in one file-scope device array of fixed size, which
// every GPU that loads this library keeps for the life of the process.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kStaticScratchBytes = size_t(64) << 20;   // 64 MiB per device
__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_static_scratch_mutex;
void *g_static_scratch_addr[kMaxDevices] = {};

}  // namespace

extern "C" size_t gb_static_scratch_bytes(void) { return kStaticScratchBytes; }

extern "C" int gb_forward_static_scratch(gb_plan *P, const float *vp, const float *rho, const float *damp,
                                         const float *wavelet, float *trace_p, float *trace_vx, float *trace_vz,
                                         float *energy_p, float *energy_vx, float *energy_vz,
                                         int32_t snapshot_every, float *snapshots, void *stream)
{
    g_last_error.clear();
    if (!P) return fail(GB_E_ARG, "null plan");
    const size_t need = gb_plan_workspace_bytes(P, 0, 0);
    if (need > kStaticScratchBytes)
        return fail(GB_E_WORKSPACE, "this model needs " + std::to_string(need) +
                                        " bytes of scratch; the static scratch holds " +
                                        std::to_string(kStaticScratchBytes) + " bytes (use gb_forward with a workspace)");
    int dev = -1;
    GB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(GB_E_ARG, "device ordinal out of range");
    void *scratch = nullptr;
    {
        // first call on this device: look the array's device address up once,
        // with this device current (the host-side symbol is not a device address)
        std::lock_guard<std::mutex> lock(g_static_scratch_mutex);
        if (!g_static_scratch_addr[dev]) {
            void *addr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&addr, g_static_scratch);
            if (e != cudaSuccess)
                return fail(GB_E_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
            g_static_scratch_addr[dev] = addr;
        }
        scratch = g_static_scratch_addr[dev];
    }
    // gb_forward clears every part of the scratch that must start at zero
    // (both wavefield time levels, the energy sums, the status word)
    return gb_forward(P, vp, rho, damp, wavelet, trace_p, trace_vx, trace_vz, energy_p, energy_vx, energy_vz,
                      snapshot_every, snapshots, nullptr, 0, GB_CKPT_F32, scratch, kStaticScratchBytes, stream);
}
