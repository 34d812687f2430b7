// C ABI of the B200 acoustic propagator (declared in include/geobrain_b200.h):
// plans, workspace layout, TMA descriptors and the host-side time loops.
#include "gb_host.h"
#include "gb_kernels.h"
#include "gb_symcache.h"

#include "gb_adj.cuh"
#include "gb_aux.cuh"
#include "gb_batch.cuh"
#include "gb_misfit.cuh"
#include "gb_stream.cuh"
#include "gb_fwd.cuh"
#include "gb_cpml_adj.cuh"
#include "gb_resident.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using namespace gb;
using gb::host::align256;
using gb::host::aligned_ws;
using gb::host::fail;
using namespace gb::host;

namespace {
thread_local std::string g_last_error;   // gb_last_error(): the message of this thread's last failure
}  // namespace

int gb::host::fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

void gb::host::clear_error() { g_last_error.clear(); }

namespace {

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

}  // namespace

int gb::host::tensor_map_encoder(PFN_cuTensorMapEncodeTiled_v12000 *out) { return get_encoder(out); }

namespace {

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

// 2-D map over one coefficient plane [Nz][pitch] fp32 (valid extent Nx).
int make_map2d(CUtensorMap *map, const float *base, int Nx, int Nz, int pitch, int box_x, int box_z)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc;
    if (int rc = get_encoder(&enc)) return rc;
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (pitch % 4)) return fail(GB_E_ARG, "coefficient plane not aligned");
    cuuint64_t dims[2] = {(cuuint64_t)Nx, (cuuint64_t)Nz};
    cuuint64_t strides[1] = {(cuuint64_t)pitch * 4};
    cuuint32_t box[2] = {(cuuint32_t)box_x, (cuuint32_t)box_z};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(GB_E_CUDA, "cuTensorMapEncodeTiled (2-D) failed (" + std::to_string((int)r) + ")");
    return GB_OK;
}


}  // namespace

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------
struct gb_plan {
    gb_model_desc d{};
    int R = 2, fs = 1;
    int Nz = 0, Nx = 0, pitch = 0;
    long long plane = 0;
    int tz = 16, spc = 0;   // tile rows, shots per CTA (0 = automatic)
    int tiles_x = 0, tiles_z = 0, n_tiles = 0, n_groups = 0;
    bool group_streams = true;                     // run shot groups on their own streams
    // Order of the tile kernels' CTAs (gb_plan_set_schedule).  0 (default):
    // blockIdx order; 1: the tiles that take the slow path first, and the
    // forward's last items split into fewer shots, so the last wave of a
    // step is short (measured no faster: 135.5 against 134.5 µs per
    // 32-shot forward step, the adjoint unchanged).
    int sched = 0;
    std::vector<int4> sched_items;                 // forward work lists, one per launch configuration
    std::vector<int> sched_off, sched_cnt;         // configuration g < n_groups: group g alone; n_groups: all
    std::vector<int> tile_order;                   // the tiles, slow path first
    std::vector<long long> sched_key;              // what the lists were built for
    int4 *d_items = nullptr;                       // this call's workspace copies (null: blockIdx order)
    int *d_tile_order = nullptr;
    float c[4] = {0, 0, 0, 0};
    std::vector<int> src_z, src_x, rcv_z, rcv_x;   // padded
    std::vector<int> rcv_ptr;                      // CSR over tiles (own receivers)
    std::vector<int4> rcv_ent;
    std::vector<int> arcv_ptr;                     // CSR over tiles: receivers inside the
    std::vector<int4> arcv_ent;                    // loaded halo rectangles (adjoint)
    // one stream per shot group (created on first use, per device)
    int stream_dev = -1;
    std::vector<cudaStream_t> gstream;
    std::vector<cudaEvent_t> gjoin;
    cudaEvent_t gfork = nullptr;
    // optional phase profiling: event pairs recorded on the caller's stream
    bool prof = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[3];   // forward, recompute, adjoint
    long long launches = 0;
    long long phase_steps[3] = {0, 0, 0};                     // time steps run per phase
    // plain forward as replays of a CUDA graph of graph_steps steps (0 = off)
    int graph_steps = 16;
    // forward steps by the streaming kernel (gb_stream.cuh): off, or on with
    // stream_chunks 16-row chunks per z-segment (0 = automatic)
    bool stream = false;
    int stream_chunks = 0;
    bool stream_usable() const { return stream && !d.free_surface && tz == 16 && !cpml; }
    // CPML absorbing layers in place of the damping (gb_plan_set_absorbing):
    // profiles [bz, az, bz_half, az_half][Nz] + [bx, ax, bx_half, ax_half][pitch]
    bool cpml = false;
    float cpml_vmax = 0.f;
    std::vector<float> cpml_prof;
    int4 cpml_still{0, 0, 0, 0};   // rows [x, y] x cols [z, w] where the profiles vanish
    int seg_chunks() const
    {
        if (stream_chunks > 0) return stream_chunks;
        // enough segments for four waves of two CTAs per SM over all shots
        const long long want = 4LL * 2 * 148;
        const long long per_seg = (long long)tiles_x * d.n_shots;
        const int n_seg = (int)std::max<long long>(1, (want + per_seg - 1) / per_seg);
        return std::max(2, (tiles_z + n_seg - 1) / n_seg);
    }
    cudaStream_t cap_stream = nullptr;                         // capture origin (never the legacy stream)
    cudaGraphExec_t gexec = nullptr;
    std::vector<uintptr_t> gkey;                               // what the instantiated graph baked in
    // CUDA graphs of chunks of gradient steps (each with what it baked in):
    // the forward steps that keep their imaging fields, the adjoint steps
    // over them, and the batched forward / adjoint steps (on a batch's first plan)
    struct GraphSlot {
        cudaGraphExec_t exec = nullptr;
        std::vector<uintptr_t> key;
        void release()
        {
            if (exec) cudaGraphExecDestroy(exec);
            exec = nullptr;
            key.clear();
        }
    };
    GraphSlot g_fwd_img, g_adj, g_batch_fwd, g_batch_adj;
    long long api_launches = 0;                                // host launch calls (kernels and graph replays)

    ~gb_plan()
    {
        clear_events();
        release_graph();
        release_streams();
    }
    void release_graph()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        gexec = nullptr;
        gkey.clear();
        g_fwd_img.release();
        g_adj.release();
        g_batch_fwd.release();
        g_batch_adj.release();
    }
    void release_streams()
    {
        release_graph();            // it references these streams' events
        if (cap_stream) cudaStreamDestroy(cap_stream);
        cap_stream = nullptr;
        for (auto s : gstream) cudaStreamDestroy(s);
        for (auto e : gjoin) cudaEventDestroy(e);
        if (gfork) cudaEventDestroy(gfork);
        gstream.clear();
        gjoin.clear();
        gfork = nullptr;
        stream_dev = -1;
    }
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
    // record the start (end) of a phase on the caller's stream
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
        const int use_spc = spc > 0 ? spc : default_spc();
        n_groups = (d.n_shots + use_spc - 1) / use_spc;
        spc_eff = use_spc;
        // (tile, (row in tile, col in tile, receiver, what)): what = 1 records
        // p and vx, 2 records vz, 3 both.  A receiver in row fs-1 under a
        // free surface records vz after the mirror vz[fs-1] = vz[fs]
        // (acoustic_2d.py:268-274), i.e. vz of row fs, which the tile that
        // owns row fs updates in the same step: its vz entry goes there.
        std::vector<std::pair<int, int4>> ents;
        for (int r = 0; r < d.n_rcv; ++r) {
            const int z = rcv_z[r], x = rcv_x[r], bx = x / TX;
            const bool split = d.free_surface && z == fs - 1;
            ents.push_back({(z / tz) * tiles_x + bx, int4{z - (z / tz) * tz, x - bx * TX, r, split ? 1 : 3}});
            if (split) ents.push_back({((z + 1) / tz) * tiles_x + bx, int4{z + 1 - ((z + 1) / tz) * tz, x - bx * TX, r, 2}});
        }
        rcv_ptr.assign(n_tiles + 1, 0);
        for (const auto &e : ents) rcv_ptr[e.first + 1]++;
        for (int t = 0; t < n_tiles; ++t) rcv_ptr[t + 1] += rcv_ptr[t];
        rcv_ent.assign(ents.size(), int4{0, 0, 0, 0});
        std::vector<int> fill(rcv_ptr.begin(), rcv_ptr.end() - 1);
        for (const auto &e : ents) rcv_ent[fill[e.first]++] = e.second;
        // adjoint: every tile whose halo rectangles [z0-2R, z0+tz+2R) x
        // [x0-8, x0+TX+8) contain the receiver injects it into its copy
        arcv_ptr.assign(n_tiles + 1, 0);
        arcv_ent.clear();
        std::vector<std::vector<int4>> per(n_tiles);
        for (int r = 0; r < d.n_rcv; ++r) {
            const int z = rcv_z[r], x = rcv_x[r];
            // rows whose adjoint takes this receiver's sources: its own, or,
            // in the mirror row fs-1 under a free surface, rows fs and fs+1
            const int zl = z, zh = (d.free_surface && z == fs - 1) ? z + 2 : z;
            // candidate tiles (a superset; the test below is exact)
            const int tz_lo = std::max(0, (zl - 2 * R) / tz - 1), tz_hi = std::min(tiles_z - 1, (zh + 2 * R) / tz + 1);
            const int tx_lo = std::max(0, (x - 8) / TX - 1), tx_hi = std::min(tiles_x - 1, (x + 8) / TX + 1);
            for (int a = tz_lo; a <= tz_hi; ++a)
                for (int b = tx_lo; b <= tx_hi; ++b) {
                    const int z0 = a * tz, x0 = b * TX;
                    if (zh >= z0 - 2 * R && zl < z0 + tz + 2 * R && x >= x0 - 8 && x < x0 + TX + 8)
                        per[a * tiles_x + b].push_back(int4{z, x, r, 0});
                }
        }
        for (int t = 0; t < n_tiles; ++t) {
            arcv_ptr[t + 1] = arcv_ptr[t] + (int)per[t].size();
            arcv_ent.insert(arcv_ent.end(), per[t].begin(), per[t].end());
        }
        res_choose();
    }
    int spc_eff = 1;

    // Resident forward (gb_resident.cuh, gb_resident_sx.cuh): -1 automatic,
    // 0 off, 1 on with the exchange through global memory after the p and
    // the v updates, 2 on with the exchange through distributed shared
    // memory in one cluster per shot, 3 on with one exchange a step through
    // global memory (4th order, no free surface); the tile rows asked for
    // (0 = automatic) and in use (0 = the tile kernel runs)
    int res_mode = -1, res_tz_req = 0, res_tz = 0;
    bool res_cluster = false, res_single = false;                      // the exchange in use
    int res_exchange() const { return res_cluster ? 1 : res_single ? 2 : 0; }
    static constexpr int kMaxClusterTiles = 16;                        // CTAs of one (non-portable) cluster
    int res_tiles_x = 0, res_tiles_z = 0, res_n = 0, res_shots = 0;   // tiling; shots per cooperative launch
    std::vector<int> res_ptr;                                          // CSR over resident tiles
    std::vector<int4> res_ent;

    // Can a resident tiling of tz rows run: enough SMs for one shot's tiles,
    // and, with a free surface, rows fs-1 .. fs+1 inside one tile (the
    // mirror rows are set where their source rows live).
    bool res_fits(int tz, int sms) const
    {
        const int tx = (Nx + TX - 1) / TX, tzn = (Nz + tz - 1) / tz;
        if ((long long)tx * tzn > sms) return false;
        if (d.free_surface && (fs - 1) / tz != (fs + 1) / tz) return false;
        return true;
    }
    // Choose the resident tiling.  Automatic mode runs it when every shot's
    // tiles fit on the SMs at once (few shots or a small grid: the cases
    // where the per-step tile kernel is launch- and latency-bound), with the
    // two exchanges through global memory and the smallest tile height that
    // fits (the most CTAs).  The cluster exchange (16 CTAs a shot at most)
    // and one exchange a step (which sends twice the cells to eight
    // neighbours and updates p on twice the rows) measured no faster on the
    // 100 x 200 grid; they run when asked for.  More shots keep the tile
    // kernel.
    bool res_single_ok() const { return R == 2 && !d.free_surface; }
    void res_choose()
    {
        res_tz = 0;
        res_cluster = res_single = false;
        if (res_mode == 0 || cpml) return;
        const int sms = sm_count();
        int best = 0;
        // passes: one exchange a step, two through global memory, cluster
        for (int pass = 0; pass < 3 && !best; ++pass) {
            const bool sx = pass == 0, cl = pass == 2;
            if (sx && !(res_single_ok() && res_mode == 3)) continue;
            if (pass == 1 && !(res_mode < 0 || res_mode == 1)) continue;
            if (cl && res_mode != 2) continue;
            for (int tz : kResidentRows) {
                if (res_tz_req && tz != res_tz_req) continue;
                if (!res_fits(tz, sms)) continue;
                const long long n = (long long)((Nx + TX - 1) / TX) * ((Nz + tz - 1) / tz);
                if (cl && n > kMaxClusterTiles) continue;
                if (res_mode < 0 && n * d.n_shots > sms) continue;
                best = tz;
                res_cluster = cl;
                res_single = sx;
                break;
            }
        }
        if (!best) return;
        res_tz = best;
        res_tiles_x = (Nx + TX - 1) / TX;
        res_tiles_z = (Nz + best - 1) / best;
        res_n = res_tiles_x * res_tiles_z;
        // clusters never wait on each other: one launch takes every shot
        res_shots = res_cluster ? d.n_shots : std::max(1, std::min(d.n_shots, sms / res_n));
        res_ptr.assign(res_n + 1, 0);
        for (int r = 0; r < d.n_rcv; ++r) res_ptr[(rcv_z[r] / best) * res_tiles_x + rcv_x[r] / TX + 1]++;
        for (int t = 0; t < res_n; ++t) res_ptr[t + 1] += res_ptr[t];
        res_ent.assign(d.n_rcv, int4{0, 0, 0, 0});
        std::vector<int> fill(res_ptr.begin(), res_ptr.end() - 1);
        for (int r = 0; r < d.n_rcv; ++r) {
            const int t = (rcv_z[r] / best) * res_tiles_x + rcv_x[r] / TX;
            res_ent[fill[t]++] = int4{rcv_z[r] - (rcv_z[r] / best) * best, rcv_x[r] - (rcv_x[r] / TX) * TX, r, 0};
        }
    }
    // SMs of the current device (148 on a B200; also the answer without one)
    static int sm_count()
    {
        int dev = 0, n = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) {
            cudaGetLastError();
            return 148;
        }
        return n;
    }

    // Enough CTAs to fill the GPU several times over, as few groups as that
    // allows (each group re-reads the coefficient tiles and adds its own
    // energy / gradient partial sums); at most 8 shots per CTA.
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
        g.n_shots = d.n_shots; g.shots_per_cta = spc_eff; g.n_groups = n_groups;
        g.nt = d.nt; g.n_rcv = d.n_rcv;
        g.dt = d.dt;
        for (int k = 0; k < 4; ++k) g.c[k] = c[k];
        g.plane = plane;
        return g;
    }

    int group_first(int grp) const { return grp * spc_eff; }
    int group_shots(int grp) const { return std::min(d.n_shots - grp * spc_eff, spc_eff); }
};

namespace {

// Workspace layout (offsets in bytes from the 256-aligned base).
struct Layout {
    size_t err, coef, fields, energy, src, rcv_ptr, rcv_ent, tile_fast, sched, amax, cpml, psi, total;
    size_t res_ptr, res_ent, res_x;           // resident forward: receiver CSR, exchange strips
    // gradient only
    size_t mu, img, g1, c1, g2, c2, arcv_ptr, arcv_ent, cprcv, cpcoef;
    int n_img;
};

size_t img_esize(int f);

// Room for the CTA schedule: the forward's work lists (each item split at
// most once, for every group alone and for all groups together) and the
// tile order.
size_t sched_bytes(const gb_plan *p)
{
    return (size_t)p->n_tiles * (4 * (size_t)std::max(p->n_groups, 1) * 16 + 4);
}

// with_gradient: 0 forward only, 1 velocity gradient, 2 velocity and density;
// checkpoint_every: steps of the recompute segment buffer, whose imaging
// fields are stored in img_fmt.
Layout layout(const gb_plan *p, int with_gradient = 0, int checkpoint_every = 0, int img_fmt = GB_IMG_F32)
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
    L.rcv_ent = o; o = align256(o + std::max<size_t>(p->rcv_ent.size(), 1) * 16);
    L.tile_fast = o; o = align256(o + (size_t)p->n_tiles * 4);
    L.sched = o; o = align256(o + sched_bytes(p));
    L.amax = o; o = align256(o + S * 3 * 4);
    if (p->cpml) {
        L.cpml = o; o = align256(o + (4 * (size_t)p->Nz + 4 * (size_t)p->pitch) * 4);
        L.psi = o; o = align256(o + 2 * S * 4 * p->plane * 4);   // two levels of the memory variables
    }
    if (p->res_tz > 0 && with_gradient == 0) {
        const ResidentKernel k = resident_kernel(p->R, p->res_tz, p->res_single ? 2 : 0);
        L.res_ptr = o; o = align256(o + (p->res_n + 1) * 4);
        L.res_ent = o; o = align256(o + std::max<size_t>(p->d.n_rcv, 1) * 16);
        L.res_x = o; o = align256(o + S * p->res_n * k.tile_words * 8);
    }
    L.n_img = with_gradient >= 2 ? 3 : 1;
    if (with_gradient > 0) {
        const size_t K = std::max(1, std::min(checkpoint_every, p->d.nt));
        const size_t G = p->n_groups;
        // adjoint state: p, vx, vz (and, with CPML, the four memory variables)
        L.mu = o; o = align256(o + S * (p->cpml ? kCpmlPlanes : 2 * 3) * p->plane * 4);
        L.img = o; o = align256(o + K * L.n_img * S * p->plane * img_esize(img_fmt));
        L.g1 = o; o = align256(o + G * p->plane * 4);
        L.c1 = o; o = align256(o + G * p->plane * 4);
        if (with_gradient >= 2) {
            L.g2 = o; o = align256(o + G * p->plane * 4);
            L.c2 = o; o = align256(o + G * p->plane * 4);
        }
        L.arcv_ptr = o; o = align256(o + (p->n_tiles + 1) * 4);
        L.arcv_ent = o; o = align256(o + std::max<size_t>(p->arcv_ent.size(), 1) * 16);
        if (p->cpml) {
            L.cprcv = o; o = align256(o + std::max<size_t>(p->d.n_rcv, 1) * 8);
            L.cpcoef = o; o = align256(o + (size_t)kCpmlCoefPlanes * p->plane * 4);
        }
    }
    L.total = o;
    return L;
}

// The plan's forward step kernel: the streaming one when the plan asks for it
// (no free surface, 16-row tiles), else the tile kernel.
StepKernel fwd_kernel(int R, int tz, bool fs, bool en, int im)
{
    if (R == 2) return fwd_tile_kernel_r2(tz, fs, en, im);
    if (R == 4) return fwd_tile_kernel_r4(tz, fs, en, im);
    return StepKernel{};
}

StepKernel fwd_kernel_for(const gb_plan *P, bool en, int im)
{
    if (P->stream_usable()) return fwd_stream_kernel_for(P->R, en, im);
    return fwd_kernel(P->R, P->tz, P->d.free_surface != 0, en, im);
}

StepKernel adj_kernel(int R, int tz, bool fs, bool rho, int img_fmt)
{
    if (R == 2) return adj_tile_kernel_r2(tz, fs, rho, img_fmt);
    if (R == 4) return adj_tile_kernel_r4(tz, fs, rho, img_fmt);
    return StepKernel{};
}

int prepare_kernel(const StepKernel &k)
{
    if (!k.fn) return fail(GB_E_UNSUPPORTED, "no kernel for this configuration");
    GB_CUDA(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem));
    return GB_OK;
}

int box_rows_p(int R, int tz) { return tz + 2 * R; }
int box_rows_vz(int R, int tz) { return tz + 4 * R; }

struct Maps {
    CUtensorMap p, vx, vz, a1, a2;
    CUtensorMap sp, svx, svz, sa1, sa2;   // 16-row blocks for the streaming kernel (when the plan uses it)
};

// Field maps over one state buffer plus the a1 / a2 coefficient maps.
int make_maps(const gb_plan *P, const float *buf, const float *a1, const float *a2, Maps *m)
{
    const int n_planes = 3 * P->d.n_shots;
    if (int rc = make_map(&m->p, buf, P->Nx, P->Nz, P->pitch, n_planes, RW, box_rows_p(P->R, P->tz))) return rc;
    if (int rc = make_map(&m->vx, buf, P->Nx, P->Nz, P->pitch, n_planes, VXW, box_rows_p(P->R, P->tz))) return rc;
    if (int rc = make_map(&m->vz, buf, P->Nx, P->Nz, P->pitch, n_planes, RW, box_rows_vz(P->R, P->tz))) return rc;
    if (int rc = make_map2d(&m->a1, a1, P->Nx, P->Nz, P->pitch, RW, box_rows_p(P->R, P->tz))) return rc;
    if (P->stream_usable()) {
        if (int rc = make_map(&m->sp, buf, P->Nx, P->Nz, P->pitch, n_planes, RW, SCH)) return rc;
        if (int rc = make_map(&m->svx, buf, P->Nx, P->Nz, P->pitch, n_planes, VXW, SCH)) return rc;
        if (int rc = make_map(&m->svz, buf, P->Nx, P->Nz, P->pitch, n_planes, RW, SCH)) return rc;
        if (int rc = make_map2d(&m->sa1, a1, P->Nx, P->Nz, P->pitch, RW, SCH)) return rc;
        if (int rc = make_map2d(&m->sa2, a2, P->Nx, P->Nz, P->pitch, RW, SCH)) return rc;
    }
    return make_map2d(&m->a2, a2, P->Nx, P->Nz, P->pitch, RW, P->tz);
}

// Per-tile fast-path flags (needs the coefficient planes).
int launch_tile_flags(gb_plan *P, const StepGeom &g, const float *k1, const float *k2, const float *k3, int *flags,
                      cudaStream_t st)
{
    const int4 still = P->cpml ? P->cpml_still : int4{-(1 << 24), 1 << 24, -(1 << 24), 1 << 24};
    if (P->R == 2 && P->tz == 16) tile_fast_kernel<2, 16><<<P->n_tiles, 256, 0, st>>>(g, k1, k2, k3, flags, still);
    if (P->R == 2 && P->tz == 32) tile_fast_kernel<2, 32><<<P->n_tiles, 256, 0, st>>>(g, k1, k2, k3, flags, still);
    if (P->R == 4 && P->tz == 16) tile_fast_kernel<4, 16><<<P->n_tiles, 256, 0, st>>>(g, k1, k2, k3, flags, still);
    if (P->R == 4 && P->tz == 32) tile_fast_kernel<4, 32><<<P->n_tiles, 256, 0, st>>>(g, k1, k2, k3, flags, still);
    GB_CUDA(cudaGetLastError());
    ++P->launches;
    return GB_OK;
}

// One step kernel launch for shot groups [grp0, grp0 + grp_count).
// A step kernel launch that may overlap the previous kernel of its stream
// (programmatic dependent launch): the step kernels wait for it on the device
// (grid_dependency_wait) before they touch memory it writes, so only the
// launch and the shared-memory set-up overlap.  Measured on 400 x 1200 with
// one shot, the forward runs 6 % faster; with 32 shots nothing changes.
cudaError_t launch_pdl(const void *fn, dim3 grid, size_t smem, void **args, cudaStream_t st)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(NTHR);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

// The CTA schedule of a launch of groups [grp0, grp0 + grp_count): the
// forward takes its work list (and its length as the grid), the adjoint the
// tile order; launches of any other set of groups keep blockIdx order.
void apply_schedule(const gb_plan *P, FwdArgs &A, int grp0, int grp_count, unsigned *grid)
{
    A.items = nullptr;
    if (!P->d_items) return;
    const int c = grp_count == 1 ? grp0 : (grp0 == 0 && grp_count == P->n_groups) ? P->n_groups : -1;
    if (c < 0 || c >= (int)P->sched_cnt.size()) return;
    A.items = P->d_items + P->sched_off[c];
    *grid = (unsigned)P->sched_cnt[c];
}

void apply_schedule(const gb_plan *P, AdjArgs &A, int, int, unsigned *) { A.tile_order = P->d_tile_order; }

template <class Args>
int launch_step(gb_plan *P, const StepKernel &K, const Maps &maps, Args A, int grp0, int grp_count, cudaStream_t st)
{
    A.grp0 = grp0;
    A.grp_count = grp_count;
    unsigned grid = (unsigned)(P->n_tiles * grp_count);
    apply_schedule(P, A, grp0, grp_count, &grid);
    void *args[] = {(void *)&maps.p, (void *)&maps.vx, (void *)&maps.vz, (void *)&maps.a1, (void *)&maps.a2,
                    (void *)&A};
    GB_CUDA(launch_pdl(K.fn, dim3(grid), K.smem, args, st));
    ++P->launches;
    ++P->api_launches;
    return GB_OK;
}

// Forward launches: the tile kernel as above, or the streaming kernel over
// (strip, segment, shot) for the shots of groups [grp0, grp0 + grp_count).
int launch_step(gb_plan *P, const StepKernel &K, const Maps &maps, FwdArgs A, int grp0, int grp_count,
                cudaStream_t st)
{
    if (!K.stream) return launch_step<FwdArgs>(P, K, maps, A, grp0, grp_count, st);
    StreamArgs SA;
    SA.shot0 = P->group_first(grp0);
    SA.n_shots = std::min(P->d.n_shots, P->group_first(grp0 + grp_count)) - SA.shot0;
    SA.seg_chunks = P->seg_chunks();
    SA.n_seg = (P->tiles_z + SA.seg_chunks - 1) / SA.seg_chunks;
    void *args[] = {(void *)&maps.sp,  (void *)&maps.svx, (void *)&maps.svz, (void *)&maps.sa1,
                    (void *)&maps.sa2, (void *)&A,         (void *)&SA};
    GB_CUDA(launch_pdl(K.fn, dim3((unsigned)P->tiles_x * SA.n_seg * SA.n_shots), K.smem, args, st));
    ++P->launches;
    ++P->api_launches;
    return GB_OK;
}

// Streams the shot groups run on: the caller's stream when there is one
// group (or grouping is off), else one stream per group forked from it.
struct GroupStreams {
    gb_plan *P;
    cudaStream_t main;
    int n;            // streams in use (1 = the caller's stream only)

    cudaStream_t at(int grp) const { return n == 1 ? main : P->gstream[grp]; }
};

// want < 0: one stream per shot group when group streams are on; else
// `want` streams (the lanes of a batch)
int group_streams(gb_plan *P, cudaStream_t main, GroupStreams *gs, int want = -1)
{
    gs->P = P;
    gs->main = main;
    gs->n = want >= 0 ? std::max(1, want) : (P->group_streams && P->n_groups > 1) ? P->n_groups : 1;
    if (gs->n == 1) return GB_OK;
    int dev = -1;
    GB_CUDA(cudaGetDevice(&dev));
    if (dev != P->stream_dev || (int)P->gstream.size() < gs->n) {
        P->release_streams();
        for (int i = 0; i < gs->n; ++i) {
            cudaStream_t s;
            cudaEvent_t e;
            GB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            GB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            P->gstream.push_back(s);
            P->gjoin.push_back(e);
        }
        GB_CUDA(cudaEventCreateWithFlags(&P->gfork, cudaEventDisableTiming));
        P->stream_dev = dev;
    }
    return GB_OK;
}

int fork(const GroupStreams &gs)
{
    if (gs.n == 1) return GB_OK;
    GB_CUDA(cudaEventRecord(gs.P->gfork, gs.main));
    for (int i = 0; i < gs.n; ++i) GB_CUDA(cudaStreamWaitEvent(gs.P->gstream[i], gs.P->gfork, 0));
    return GB_OK;
}

int join(const GroupStreams &gs)
{
    if (gs.n == 1) return GB_OK;
    for (int i = 0; i < gs.n; ++i) {
        GB_CUDA(cudaEventRecord(gs.P->gjoin[i], gs.P->gstream[i]));
        GB_CUDA(cudaStreamWaitEvent(gs.main, gs.P->gjoin[i], 0));
    }
    return GB_OK;
}

// groups handled by one launch on stream i: all of them on a single stream
inline void launch_groups(const GroupStreams &gs, int i, int n_groups, int *g0, int *gc)
{
    if (gs.n == 1) {
        *g0 = 0;
        *gc = n_groups;
    } else {
        *g0 = i;
        *gc = 1;
    }
}

// ---------------------------------------------------------------------------
// CUDA graph of a chunk of plain forward steps.  The graph holds C steps of
// every shot group (C even, so step j of the chunk reads state level j & 1)
// with the group fork / join, then advances a device step counter by C; the
// step kernels take their step index from that counter.  It is captured once
// for a given set of buffers and replayed nt / C times.
// ---------------------------------------------------------------------------
constexpr int kMaxGraphSteps = 64;

int capture_forward_chunk(gb_plan *P, const StepKernel &K, const Maps (&maps)[2], float *const (&buf)[2],
                          float *const (&psi)[2], FwdArgs A, int C, int *step_ctr, cudaGraphExec_t *out)
{
    GroupStreams gs;
    if (int rc = group_streams(P, nullptr, &gs)) return rc;      // (re)creating the group streams drops cap_stream
    if (!P->cap_stream) GB_CUDA(cudaStreamCreateWithFlags(&P->cap_stream, cudaStreamNonBlocking));
    gs.main = P->cap_stream;
    const long long launches = P->launches;
    GB_CUDA(cudaStreamBeginCapture(P->cap_stream, cudaStreamCaptureModeThreadLocal));
    int rc = fork(gs);
    A.step_base = step_ctr;
    for (int j = 0; j < C && rc == GB_OK; ++j) {
        A.it = j;
        A.out = buf[(j & 1) ^ 1];
        if (A.cpml) {
            A.psi_in = psi[j & 1];
            A.psi_out = psi[(j & 1) ^ 1];
        }
        for (int i = 0; i < gs.n && rc == GB_OK; ++i) {
            int g0, gc;
            launch_groups(gs, i, P->n_groups, &g0, &gc);
            rc = launch_step(P, K, maps[j & 1], A, g0, gc, gs.at(i));
        }
    }
    if (rc == GB_OK) rc = join(gs);
    if (rc == GB_OK) {
        step_advance_kernel<<<1, 1, 0, P->cap_stream>>>(step_ctr, C);
        if (cudaGetLastError() != cudaSuccess) rc = fail(GB_E_CUDA, "graph capture: launch failed");
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(P->cap_stream, &graph);   // always end the capture
    P->launches = launches;
    if (rc != GB_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ec != cudaSuccess) return fail(GB_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
    const cudaError_t ei = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return fail(GB_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    return GB_OK;
}

// Capture `C` steps of a step loop into `slot` (unless it already holds a
// graph for `key`): launch(j, gs) launches step j of the chunk on the group
// streams gs, and after the steps the device counter ctr moves by `advance`;
// the step kernels read their step index from that counter.
template <class Launch>
int capture_chunk(gb_plan *P, gb_plan::GraphSlot &slot, const std::vector<uintptr_t> &key, int C, int *ctr,
                  int advance, bool group_streams_on, Launch launch, int n_streams = -1)
{
    if (slot.exec && slot.key == key) return GB_OK;
    slot.release();
    GroupStreams gs;
    if (group_streams_on) {
        // (re)creating the group streams drops cap_stream
        if (int rc = group_streams(P, nullptr, &gs, n_streams)) return rc;
    } else {
        gs.P = P;
        gs.n = 1;
    }
    if (!P->cap_stream) GB_CUDA(cudaStreamCreateWithFlags(&P->cap_stream, cudaStreamNonBlocking));
    gs.main = P->cap_stream;
    const long long launches = P->launches, api = P->api_launches;
    GB_CUDA(cudaStreamBeginCapture(P->cap_stream, cudaStreamCaptureModeThreadLocal));
    int rc = group_streams_on ? fork(gs) : GB_OK;
    for (int j = 0; j < C && rc == GB_OK; ++j) rc = launch(j, gs);
    if (rc == GB_OK && group_streams_on) rc = join(gs);
    if (rc == GB_OK) {
        step_advance_kernel<<<1, 1, 0, P->cap_stream>>>(ctr, advance);
        if (cudaGetLastError() != cudaSuccess) rc = fail(GB_E_CUDA, "graph capture: launch failed");
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(P->cap_stream, &graph);   // always end the capture
    P->launches = launches;
    P->api_launches = api;
    if (rc != GB_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ec != cudaSuccess) return fail(GB_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
    const cudaError_t ei = cudaGraphInstantiate(&slot.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
        slot.exec = nullptr;
        return fail(GB_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    }
    slot.key = key;
    return GB_OK;
}

// Per-checkpoint sizes of the 16-bit formats.
size_t ck16_bytes(const gb_plan *p) { return align256((size_t)p->d.n_shots * 3 * p->plane * 2); }
size_t ck_scale_bytes(const gb_plan *p) { return align256((size_t)p->d.n_shots * 3 * 4); }
size_t ck_bytes(const gb_plan *p, int fmt)
{
    if (fmt == GB_CKPT_F32) return (size_t)p->d.n_shots * 3 * p->plane * 4;
    if (fmt == GB_CKPT_F24) return align256((size_t)p->d.n_shots * 3 * p->plane * 3);
    return ck16_bytes(p) + ck_scale_bytes(p);
}

// Save shots [s0, s0 + ns) of `state` into checkpoint k.
int save_checkpoint(gb_plan *P, const float *state, void *ckpts, int k, int fmt, unsigned int *amax, int s0, int ns,
                    cudaStream_t st)
{
    const long long pl = P->plane;
    char *base = reinterpret_cast<char *>(ckpts) + (size_t)k * ck_bytes(P, fmt);
    const float *src = state + (size_t)s0 * 3 * pl;
    if (fmt == GB_CKPT_F32) {
        GB_CUDA(cudaMemcpyAsync(base + (size_t)s0 * 3 * pl * 4, src, (size_t)ns * 3 * pl * 4, cudaMemcpyDeviceToDevice,
                                st));
        return GB_OK;
    }
    if (fmt == GB_CKPT_F24) {
        // plane is a multiple of 32, so every shot's block starts on a 4-value group
        pack24_kernel<<<4 * 148, 256, 0, st>>>(src, (long long)ns * 3 * pl / 4,
                                               reinterpret_cast<float *>(base + (size_t)s0 * 3 * pl * 3));
        GB_CUDA(cudaGetLastError());
        ++P->launches;
        return GB_OK;
    }
    float *scales = reinterpret_cast<float *>(base + ck16_bytes(P)) + 3 * s0;
    unsigned int *am = amax + 3 * s0;
    GB_CUDA(cudaMemsetAsync(am, 0, (size_t)ns * 3 * 4, st));
    dim3 grid(64, ns * 3);
    plane_absmax_kernel<<<grid, 256, 0, st>>>(src, pl, am);
    if (fmt == GB_CKPT_BF16)
        pack16_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(
            src, pl, am, reinterpret_cast<__nv_bfloat16 *>(base) + (size_t)s0 * 3 * pl, scales);
    else
        pack16_kernel<__half><<<grid, 256, 0, st>>>(src, pl, am, reinterpret_cast<__half *>(base) + (size_t)s0 * 3 * pl,
                                                   scales);
    GB_CUDA(cudaGetLastError());
    P->launches += 2;
    return GB_OK;
}

int restore_checkpoint(gb_plan *P, float *state, const void *ckpts, int k, int fmt, int s0, int ns, cudaStream_t st)
{
    const long long pl = P->plane;
    const char *base = reinterpret_cast<const char *>(ckpts) + (size_t)k * ck_bytes(P, fmt);
    float *dst = state + (size_t)s0 * 3 * pl;
    if (fmt == GB_CKPT_F32) {
        GB_CUDA(cudaMemcpyAsync(dst, base + (size_t)s0 * 3 * pl * 4, (size_t)ns * 3 * pl * 4, cudaMemcpyDeviceToDevice,
                                st));
        return GB_OK;
    }
    if (fmt == GB_CKPT_F24) {
        unpack24_kernel<<<4 * 148, 256, 0, st>>>(reinterpret_cast<const float *>(base + (size_t)s0 * 3 * pl * 3),
                                                 (long long)ns * 3 * pl / 4, dst);
        GB_CUDA(cudaGetLastError());
        ++P->launches;
        return GB_OK;
    }
    const float *scales = reinterpret_cast<const float *>(base + ck16_bytes(P)) + 3 * s0;
    dim3 grid(64, ns * 3);
    if (fmt == GB_CKPT_BF16)
        unpack16_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(
            reinterpret_cast<const __nv_bfloat16 *>(base) + (size_t)s0 * 3 * pl, scales, pl, dst);
    else
        unpack16_kernel<__half><<<grid, 256, 0, st>>>(reinterpret_cast<const __half *>(base) + (size_t)s0 * 3 * pl,
                                                     scales, pl, dst);
    GB_CUDA(cudaGetLastError());
    ++P->launches;
    return GB_OK;
}

// The CTA schedule for `slots` resident CTAs of the tile kernels (every SM's
// share).  Tiles whose rectangles reach into the absorbing frame, the free
// surface or past the grid's edge take the masked, damped slow path: they go
// first.  Each tile's groups stay together.  In every forward list the last
// items (as many as the launch has resident slots) are split into two
// halves of their shots, so the launch ends on short items.
void build_schedule(gb_plan *P, int slots)
{
    const std::vector<long long> key = {P->n_tiles, P->n_groups, P->spc_eff, P->tz,     P->R,   slots,
                                        P->group_streams, P->d.n_shots, P->d.nabc, P->d.nz, P->d.nx, P->fs};
    if (key == P->sched_key) return;
    P->sched_key = key;
    const int R = P->R, TZ = P->tz, nabc = P->d.nabc;
    const int zlo = std::max(P->fs + 1, nabc), zhi = nabc + P->d.nz, xlo = nabc, xhi = nabc + P->d.nx;
    auto slow = [&](int t) {
        const int z0 = (t / P->tiles_x) * TZ, x0 = (t % P->tiles_x) * TX;
        return !(z0 - 2 * R >= zlo && z0 + TZ + 2 * R <= zhi && x0 - 8 >= xlo && x0 + TX + 8 <= xhi);
    };
    P->tile_order.clear();
    for (int pass = 0; pass < 2; ++pass)
        for (int t = 0; t < P->n_tiles; ++t)
            if (slow(t) == (pass == 0)) P->tile_order.push_back(t);
    P->sched_items.clear();
    P->sched_off.clear();
    P->sched_cnt.clear();
    const int concurrent = (P->group_streams && P->n_groups > 1) ? P->n_groups : 1;
    for (int c = 0; c <= P->n_groups; ++c) {
        const int g0 = c < P->n_groups ? c : 0, gc = c < P->n_groups ? 1 : P->n_groups;
        const int per_launch = c < P->n_groups ? std::max(1, slots / concurrent) : slots;
        std::vector<int4> it;
        for (int t : P->tile_order)
            for (int g = g0; g < g0 + gc; ++g) it.push_back(make_int4(t, P->group_first(g), P->group_shots(g), 0));
        P->sched_off.push_back((int)P->sched_items.size());
        const int n = (int)it.size(), first_split = std::max(0, n - per_launch);
        for (int i = 0; i < n; ++i) {
            const int4 w = it[i];
            if (i >= first_split && w.z >= 2) {
                const int h = w.z / 2;
                P->sched_items.push_back(make_int4(w.x, w.y, h, 0));
                P->sched_items.push_back(make_int4(w.x, w.y + h, w.z - h, 0));
            } else {
                P->sched_items.push_back(w);
            }
        }
        P->sched_cnt.push_back((int)P->sched_items.size() - P->sched_off.back());
    }
}

// Everything both passes set up: metadata upload, coefficient planes, flags.
struct Setup {
    int *err;
    float *a1, *k1, *a2, *k2, *k3;
    int *d_src, *d_rptr, *tile_fast;
    int4 *d_rent;
    unsigned int *amax;
    float *cpml = nullptr, *psi[2] = {nullptr, nullptr};
};

int common_setup(gb_plan *P, const Layout &L, char *ws, const float *vp, const float *rho, const float *damp,
                 cudaStream_t st, Setup *S)
{
    const gb_model_desc &d = P->d;
    S->err = reinterpret_cast<int *>(ws + L.err);
    float *coef = reinterpret_cast<float *>(ws + L.coef);
    S->a1 = coef;
    S->k1 = coef + P->plane;
    S->a2 = coef + 2 * P->plane;
    S->k2 = coef + 3 * P->plane;
    S->k3 = coef + 4 * P->plane;
    S->d_src = reinterpret_cast<int *>(ws + L.src);
    S->d_rptr = reinterpret_cast<int *>(ws + L.rcv_ptr);
    S->d_rent = reinterpret_cast<int4 *>(ws + L.rcv_ent);
    S->tile_fast = reinterpret_cast<int *>(ws + L.tile_fast);
    S->amax = reinterpret_cast<unsigned int *>(ws + L.amax);
    GB_CUDA(cudaMemsetAsync(S->err, 0, 4, st));
    GB_CUDA(cudaMemcpyAsync(S->d_src, P->src_z.data(), d.n_shots * 4, cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemcpyAsync(S->d_src + d.n_shots, P->src_x.data(), d.n_shots * 4, cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemcpyAsync(S->d_rptr, P->rcv_ptr.data(), (P->n_tiles + 1) * 4, cudaMemcpyHostToDevice, st));
    if (!P->rcv_ent.empty())
        GB_CUDA(cudaMemcpyAsync(S->d_rent, P->rcv_ent.data(), P->rcv_ent.size() * 16, cudaMemcpyHostToDevice, st));
    P->d_items = nullptr;
    P->d_tile_order = nullptr;
    if (P->sched) {
        int dev = 0, sms = 0;
        GB_CUDA(cudaGetDevice(&dev));
        GB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        build_schedule(P, sms * (P->tz <= 16 ? 2 : 1));
        char *sb = ws + L.sched;
        P->d_items = reinterpret_cast<int4 *>(sb);
        P->d_tile_order = reinterpret_cast<int *>(sb + P->sched_items.size() * 16);
        GB_CUDA(cudaMemcpyAsync(P->d_items, P->sched_items.data(), P->sched_items.size() * 16, cudaMemcpyHostToDevice,
                                st));
        GB_CUDA(cudaMemcpyAsync(P->d_tile_order, P->tile_order.data(), P->tile_order.size() * 4,
                                cudaMemcpyHostToDevice, st));
    }
    coef_kernel<<<4 * 148, 256, 0, st>>>(vp, rho, damp, d.nz, d.nx, d.nabc, P->Nz, P->Nx, P->pitch, P->fs, d.dt, d.dx,
                                         S->a1, S->k1, S->a2, S->k2, S->k3);
    GB_CUDA(cudaGetLastError());
    ++P->launches;
    if (P->cpml) {
        // the CPML layers replace the damping: no k terms, profiles and memory variables instead
        GB_CUDA(cudaMemsetAsync(S->k1, 0, P->plane * 4, st));       // k1, then k2 and k3 (a2 sits between)
        GB_CUDA(cudaMemsetAsync(S->k2, 0, 2 * P->plane * 4, st));
        S->cpml = reinterpret_cast<float *>(ws + L.cpml);
        S->psi[0] = reinterpret_cast<float *>(ws + L.psi);
        S->psi[1] = S->psi[0] + (size_t)d.n_shots * 4 * P->plane;
        GB_CUDA(cudaMemcpyAsync(S->cpml, P->cpml_prof.data(), P->cpml_prof.size() * 4, cudaMemcpyHostToDevice, st));
        GB_CUDA(cudaMemsetAsync(S->psi[0], 0, 2 * (size_t)d.n_shots * 4 * P->plane * 4, st));
    }
    return launch_tile_flags(P, P->geom(), S->k1, S->k2, S->k3, S->tile_fast, st);
}


bool img_format_ok(int f) { return f == GB_IMG_F32 || f == GB_IMG_BF16 || f == GB_IMG_F24; }
size_t img_esize(int f) { return f == GB_IMG_BF16 ? 2 : f == GB_IMG_F24 ? 3 : 4; }
static_assert(GB_IMG_F32 == kImgF32 && GB_IMG_BF16 == kImgBF16 && GB_IMG_F24 == kImgF24,
              "imaging format codes of the header and the kernels agree");

// Element `e` of an imaging buffer whose elements are esize bytes, as the
// float pointer the kernels take (they widen the short formats themselves).
float *img_at(void *base, size_t e, size_t esize)
{
    return reinterpret_cast<float *>(reinterpret_cast<char *>(base) + e * esize);
}

int check_store(const gb_plan *P, const gb_grad_store *store)
{
    if (!store) return GB_OK;
    if (store->checkpoint_every < 1) return fail(GB_E_ARG, "checkpoint_every must be >= 1");
    if (store->format < GB_CKPT_F32 || store->format > GB_CKPT_F24) return fail(GB_E_ARG, "unknown checkpoint format");
    if (store->cached_steps < 0 || store->cached_steps > P->d.nt) return fail(GB_E_ARG, "cached_steps out of range");
    if (store->cached_steps > 0 && !store->imaging) return fail(GB_E_ARG, "cached_steps > 0 needs an imaging buffer");
    if (!img_format_ok(store->imaging_format))
        return fail(GB_E_ARG, "imaging_format must be GB_IMG_F32, GB_IMG_BF16 or GB_IMG_F24");
    if (store->cached_steps < P->d.nt && !store->checkpoints) return fail(GB_E_ARG, "checkpoint storage missing");
    return GB_OK;
}

// Plain forward by the resident kernel: cooperative launches of res_n tiles x
// res_shots shots, each running a chunk of steps with the state in shared
// memory (chunks end where a snapshot of shot 0 is due).  The state starts
// and ends in buf (level 0 of the workspace's fields).
int forward_resident(gb_plan *P, const Layout &L, char *ws, const Setup &Su, float *buf, float *energy,
                     bool want_energy, const float *wavelet, float *trace_p, float *trace_vx, float *trace_vz,
                     int32_t snapshot_every, float *snapshots, cudaStream_t st)
{
    const gb_model_desc &d = P->d;
    const int S = d.n_shots;
    const ResidentKernel K = resident_kernel(P->R, P->res_tz, P->res_exchange());
    if (!K.fn) return fail(GB_E_UNSUPPORTED, "no resident kernel for this tile height");
    GB_CUDA(cudaFuncSetAttribute(K.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K.smem));
    if (P->res_cluster && P->res_n > 8) GB_CUDA(cudaFuncSetAttribute(K.fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    int *d_ptr = reinterpret_cast<int *>(ws + L.res_ptr);
    int4 *d_ent = reinterpret_cast<int4 *>(ws + L.res_ent);
    GB_CUDA(cudaMemcpyAsync(d_ptr, P->res_ptr.data(), (P->res_n + 1) * 4, cudaMemcpyHostToDevice, st));
    if (d.n_rcv) GB_CUDA(cudaMemcpyAsync(d_ent, P->res_ent.data(), d.n_rcv * 16, cudaMemcpyHostToDevice, st));
    // the strips' tags start at 0, which no step's tag is
    if (!P->res_cluster)
        GB_CUDA(cudaMemsetAsync(ws + L.res_x, 0, (size_t)S * P->res_n * K.tile_words * 8, st));
    ResArgs A{};
    A.g = P->geom();
    A.tiles_x = P->res_tiles_x;
    A.tiles_z = P->res_tiles_z;
    A.n_tiles = P->res_n;
    A.energy = want_energy ? 1 : 0;
    A.free_surface = d.free_surface ? 1 : 0;
    A.a1 = Su.a1; A.k1 = Su.k1; A.a2 = Su.a2; A.k2 = Su.k2; A.k3 = Su.k3;
    A.state = buf;
    A.src_z = Su.d_src; A.src_x = Su.d_src + S;
    A.wavelet = wavelet;
    A.rcv_ptr = d_ptr; A.rcv_ent = d_ent;
    A.tr_p = trace_p; A.tr_vx = trace_vx; A.tr_vz = trace_vz;
    A.energy_map = want_energy ? energy : nullptr;
    A.xbuf = reinterpret_cast<uint2 *>(ws + L.res_x);
    A.err = Su.err;
    int snap_i = 0;
    for (int s0 = 0; s0 < S; s0 += P->res_shots) {
        const int ns = std::min(P->res_shots, S - s0);
        A.shot0 = s0;
        const bool snaps = s0 == 0 && snapshot_every > 0 && snapshots;
        for (int it0 = 0; it0 < d.nt;) {
            const int it1 = snaps ? std::min(d.nt, (it0 / snapshot_every + 1) * snapshot_every) : d.nt;
            A.it0 = it0;
            A.it1 = it1;
            void *args[] = {(void *)&A};
            if (P->res_cluster) {
                // one cluster of res_n CTAs per shot (cluster rank = tile)
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3((unsigned)(P->res_n * ns));
                cfg.blockDim = dim3(K.threads);
                cfg.dynamicSmemBytes = K.smem;
                cfg.stream = st;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeClusterDimension;
                attr[0].val.clusterDim.x = (unsigned)P->res_n;
                attr[0].val.clusterDim.y = 1;
                attr[0].val.clusterDim.z = 1;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                int n_clusters = 0;
                GB_CUDA(cudaOccupancyMaxActiveClusters(&n_clusters, K.fn, &cfg));
                if (n_clusters < 1)
                    return fail(GB_E_UNSUPPORTED, "this device cannot schedule a cluster of " +
                                                      std::to_string(P->res_n) + " resident tiles");
                GB_CUDA(cudaLaunchKernelExC(&cfg, K.fn, args));
            } else {
                GB_CUDA(cudaLaunchCooperativeKernel(K.fn, dim3((unsigned)(P->res_n * ns)), dim3(K.threads), args,
                                                    K.smem, st));
            }
            ++P->launches;
            ++P->api_launches;
            if (snaps) {
                GB_CUDA(cudaMemcpy2DAsync(snapshots + (size_t)snap_i * d.nz * d.nx, (size_t)d.nx * 4,
                                          buf + (size_t)d.nabc * P->pitch + d.nabc, (size_t)P->pitch * 4,
                                          (size_t)d.nx * 4, d.nz, cudaMemcpyDeviceToDevice, st));
                ++snap_i;
            }
            it0 = it1;
        }
    }
    return GB_OK;
}

// Gradient of a CPML plan: the adjoint sweep of gb_cpml_adj.cuh over every
// step, from imaging fields the forward kept for all nt steps (no recompute,
// so no memory variables need checkpointing).
int backward_cpml(gb_plan *P, const float *vp, const float *rho, const float *damp, const float *res_p,
                  const float *res_vx, const float *res_vz, const gb_grad_store *store, float *grad_vp,
                  float *grad_rho, float *grad_wavelet, void *workspace, size_t workspace_bytes, cudaStream_t st)
{
    const gb_model_desc &d = P->d;
    if (store->cached_steps < d.nt)
        return fail(GB_E_UNSUPPORTED, "CPML gradients need every step's imaging fields in the store (cached_steps = nt)");
    const bool rho_fields = store->with_rho != 0;
    const int ifmt = store->imaging_format;
    const Layout L = layout(P, rho_fields ? 2 : 1, 1, ifmt);
    char *ws = aligned_ws(workspace);
    if (!workspace || workspace_bytes < L.total + (size_t)(ws - reinterpret_cast<char *>(workspace)))
        return fail(GB_E_WORKSPACE, "workspace too small");
    Setup Su;
    if (int rc = common_setup(P, L, ws, vp, rho, damp, st, &Su)) return rc;
    const int S = d.n_shots;
    float *lam = reinterpret_cast<float *>(ws + L.mu);   // [S][kCpmlPlanes][plane]
    float *G1 = reinterpret_cast<float *>(ws + L.g1), *C1 = reinterpret_cast<float *>(ws + L.c1);
    float *G2 = rho_fields ? reinterpret_cast<float *>(ws + L.g2) : nullptr;
    float *C2 = rho_fields ? reinterpret_cast<float *>(ws + L.c2) : nullptr;
    GB_CUDA(cudaMemsetAsync(lam, 0, (size_t)S * kCpmlPlanes * P->plane * 4, st));
    GB_CUDA(cudaMemsetAsync(G1, 0, (size_t)P->n_groups * P->plane * 4, st));
    GB_CUDA(cudaMemsetAsync(C1, 0, (size_t)P->n_groups * P->plane * 4, st));
    if (G2) {
        GB_CUDA(cudaMemsetAsync(G2, 0, (size_t)P->n_groups * P->plane * 4, st));
        GB_CUDA(cudaMemsetAsync(C2, 0, (size_t)P->n_groups * P->plane * 4, st));
    }
    int2 *d_rcv = reinterpret_cast<int2 *>(ws + L.cprcv);
    std::vector<int2> hr(d.n_rcv);
    for (int r = 0; r < d.n_rcv; ++r) hr[r] = make_int2(P->rcv_z[r], P->rcv_x[r]);
    // pageable host vector: cudaMemcpyAsync copies it before returning
    if (d.n_rcv) GB_CUDA(cudaMemcpyAsync(d_rcv, hr.data(), hr.size() * 8, cudaMemcpyHostToDevice, st));

    const StepGeom g = P->geom();
    float *cpcoef = reinterpret_cast<float *>(ws + L.cpcoef);
    cpml_adj_coef_kernel<<<4 * 148, 256, 0, st>>>(g, Su.a1, Su.a2, Su.cpml, cpcoef);
    ++P->launches;
    CpmlAdjArgs4 A{};
    A.g = g;
    A.a1 = Su.a1;
    A.a2 = Su.a2;
    A.cp = cpcoef;
    A.lam = lam;
    A.img_field_stride = (long long)S * P->plane;
    A.img_fmt = ifmt;
    A.G1 = G1; A.C1 = C1; A.G2 = G2; A.C2 = C2;
    const bool fs = d.free_surface != 0;
    A.free_surface = fs;
    const bool inject = d.n_rcv > 0 && (res_p || res_vx || res_vz);
    const size_t step_img = (size_t)(rho_fields ? 3 : 1) * S * P->plane;
    const dim3 block(32, 4), grid((P->Nx + 127) / 128, (P->Nz + 4 * kCpLZ - 1) / (4 * kCpLZ), P->n_groups);
    const int fold_blocks = (int)std::min<long long>(1024, ((long long)S * P->Nx + 255) / 256);
    P->mark(2, true, st);
    P->phase_steps[2] += d.nt;
    int sv = 0, sp = 0;   // the memory-variable slots read this step
    for (int it = d.nt - 1; it >= 0; --it) {
        if (inject) {
            cpml_inject_kernel<<<std::max(1, std::min(1024, (S * d.n_rcv + 255) / 256)), 256, 0, st>>>(
                g, lam, d_rcv, res_p, res_vx, res_vz, it);
            ++P->launches;
        }
        if (fs) {
            cpml_fold_kernel<<<fold_blocks, 256, 0, st>>>(g, lam, kLamVZ, 1, 1.f);
            ++P->launches;
        }
        A.img = img_at(store->imaging, (size_t)it * step_img, img_esize(ifmt));
        A.psi_in = kPsiV0 + 2 * sv;
        A.psi_out = kPsiV0 + 2 * (sv ^ 1);
        if (P->R == 4) cpml_adj_v_kernel<4><<<grid, block, 0, st>>>(A);
        else cpml_adj_v_kernel<2><<<grid, block, 0, st>>>(A);
        sv ^= 1;
        if (fs) {
            cpml_fold_kernel<<<fold_blocks, 256, 0, st>>>(g, lam, kLamP, 2, -1.f);
            ++P->launches;
        }
        if (grad_wavelet) {
            cpml_wavelet_grad_kernel<<<(S + 127) / 128, 128, 0, st>>>(g, lam, Su.d_src, Su.d_src + S, grad_wavelet,
                                                                       it);
            ++P->launches;
        }
        A.psi_in = kPsiP0 + 2 * sp;
        A.psi_out = kPsiP0 + 2 * (sp ^ 1);
        if (P->R == 4) cpml_adj_p_kernel<4><<<grid, block, 0, st>>>(A);
        else cpml_adj_p_kernel<2><<<grid, block, 0, st>>>(A);
        sp ^= 1;
        P->launches += 2;
        GB_CUDA(cudaGetLastError());
    }
    P->mark(2, false, st);
    grad_finish_kernel<<<4 * 148, 256, 0, st>>>(vp, rho, G1, C1, G2, C2, P->n_groups, P->plane, d.nz, d.nx, d.nabc,
                                                P->pitch, grad_vp, grad_rho);
    GB_CUDA(cudaGetLastError());
    ++P->launches;
    return GB_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char *gb_last_error(void) { return g_last_error.c_str(); }

const char *gb_version(void) { return "geobrain_b200 0.2 (sm_100a)"; }

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
    p->spc = shots_per_cta ? std::min(std::min(shots_per_cta, p->d.n_shots), kMaxShotsPerCta) : 0;
    p->retile();
    p->release_graph();
    return GB_OK;
}

int gb_plan_set_resident(gb_plan *p, int mode, int tile_rows)
{
    if (!p) return fail(GB_E_ARG, "null plan");
    if (mode < -1 || mode > 3)
        return fail(GB_E_ARG, "mode must be -1 (automatic), 0 (off), 1 (global exchange), 2 (cluster exchange) "
                              "or 3 (one global exchange a step)");
    bool known = tile_rows == 0;
    for (int tz : kResidentRows) known |= tz == tile_rows;
    if (!known) return fail(GB_E_ARG, "tile_rows must be 0, 4, 8, 12, 16, 24, 32, 36 or 40");
    p->res_mode = mode;
    p->res_tz_req = tile_rows;
    p->res_choose();
    if (mode >= 1 && p->res_tz == 0) {
        p->res_mode = -1;
        p->res_tz_req = 0;
        p->res_choose();
        return fail(GB_E_UNSUPPORTED,
                    p->cpml ? "the resident forward does not run CPML plans"
                    : mode == 3 && !p->res_single_ok()
                        ? "one exchange a step needs the 4th-order scheme without a free surface"
                        : "no resident tiling of that height fits this grid on this device");
    }
    return GB_OK;
}

int gb_plan_get_resident(const gb_plan *p, int *tile_rows, int *shots_per_launch, int *cluster)
{
    if (!p) return fail(GB_E_ARG, "null plan");
    if (tile_rows) *tile_rows = p->res_tz;
    if (shots_per_launch) *shots_per_launch = p->res_tz ? p->res_shots : 0;
    if (cluster) *cluster = p->res_tz ? p->res_exchange() : 0;
    return GB_OK;
}

int gb_plan_set_group_streams(gb_plan *p, int enable)
{
    if (!p) return fail(GB_E_ARG, "null plan");
    p->group_streams = enable != 0;
    p->release_graph();
    return GB_OK;
}

int gb_plan_get_config(const gb_plan *p, int *tile_rows, int *shots_per_cta, int *group_streams, int *graph_steps,
                       int *stream_chunks)
{
    if (!p) return fail(GB_E_ARG, "null plan");
    if (tile_rows) *tile_rows = p->tz;
    if (shots_per_cta) *shots_per_cta = p->spc_eff;
    if (group_streams) *group_streams = p->group_streams ? 1 : 0;
    if (graph_steps) *graph_steps = p->graph_steps;
    if (stream_chunks) *stream_chunks = p->stream_usable() ? p->seg_chunks() : 0;
    return GB_OK;
}

int gb_plan_set_absorbing(gb_plan *p, int mode, float vmax)
{
    if (!p) return fail(GB_E_ARG, "null plan");
    if (mode != GB_ABSORB_DAMPING && mode != GB_ABSORB_CPML) return fail(GB_E_ARG, "unknown absorbing mode");
    if (mode == GB_ABSORB_CPML && !(vmax > 0.f)) return fail(GB_E_ARG, "CPML needs vmax > 0");
    if ((mode == GB_ABSORB_CPML) == p->cpml && (!p->cpml || vmax == p->cpml_vmax)) return GB_OK;   // unchanged
    p->release_graph();
    p->cpml = mode == GB_ABSORB_CPML;
    p->res_choose();   // the resident forward runs the damping layers only
    p->cpml_vmax = vmax;
    p->cpml_prof.clear();
    if (!p->cpml) return GB_OK;
    const int pml = p->d.nabc;
    if (pml < 1) return fail(GB_E_ARG, "CPML needs nabc >= 1");
    // quadratic profile d(r) = d0 r^2, r = depth into the layer / nabc, d0 for
    // a 1e-6 reflection; b = exp(-d dt), a = b - 1 (no kappa / alpha terms)
    const double d0 = -3.0 * vmax * std::log(1e-6) / (2.0 * pml * p->d.dx), dt = p->d.dt;
    auto depth = [&](double c, int N, bool lo) {
        double r = 0.0;
        if (lo && c < pml) r = (pml - c) / pml;
        else if (c > N - 1 - pml) r = (c - (N - 1 - pml)) / pml;
        return std::min(r, 1.0);
    };
    p->cpml_prof.assign(4 * (size_t)p->Nz + 4 * (size_t)p->pitch, 0.f);
    float *z = p->cpml_prof.data(), *x = z + 4 * p->Nz;
    const bool top = !p->d.free_surface;   // a free surface has no layer above it
    for (int i = 0; i < p->Nz; ++i)
        for (int h = 0; h < 2; ++h) {
            const double r = depth(i + 0.5 * h, p->Nz, top), b = std::exp(-d0 * r * r * dt);
            z[(2 * h) * p->Nz + i] = (float)b;
            z[(2 * h + 1) * p->Nz + i] = (float)(b - 1.0);
        }
    for (int j = 0; j < p->pitch; ++j)
        for (int h = 0; h < 2; ++h) {
            const double r = j < p->Nx ? depth(j + 0.5 * h, p->Nx, true) : 0.0, b = std::exp(-d0 * r * r * dt);
            x[(2 * h) * p->pitch + j] = (float)b;
            x[(2 * h + 1) * p->pitch + j] = (float)(b - 1.0);
        }
    p->cpml_still = int4{top ? pml : -(1 << 24), p->Nz - 2 - pml, pml, p->Nx - 2 - pml};
    return GB_OK;
}

int gb_plan_set_streaming(gb_plan *p, int enable, int seg_chunks)
{
    if (!p) return fail(GB_E_ARG, "null plan");
    if (seg_chunks < 0) return fail(GB_E_ARG, "seg_chunks must be >= 0");
    p->stream = enable != 0;
    p->stream_chunks = seg_chunks;
    p->release_graph();
    return GB_OK;
}

int gb_plan_set_schedule(gb_plan *p, int mode)
{
    if (!p) return fail(GB_E_ARG, "null plan");
    if (mode != 0 && mode != 1) return fail(GB_E_ARG, "schedule mode must be 0 or 1");
    p->sched = mode;
    p->release_graph();
    return GB_OK;
}

int gb_plan_schedule_items(gb_plan *p, int slots, int config, int32_t *items, int cap, int *n_items)
{
    if (!p || !n_items) return fail(GB_E_ARG, "null argument");
    if (slots < 1 || config < 0 || config > p->n_groups || cap < 0) return fail(GB_E_ARG, "invalid slots or configuration");
    build_schedule(p, slots);
    const int n = p->sched_cnt[config];
    *n_items = n;
    if (items) {
        if (cap < n) return fail(GB_E_ARG, "item buffer too small");
        const int4 *src = p->sched_items.data() + p->sched_off[config];
        for (int i = 0; i < n; ++i) {
            items[3 * i] = src[i].x;
            items[3 * i + 1] = src[i].y;
            items[3 * i + 2] = src[i].z;
        }
    }
    return GB_OK;
}

int gb_plan_set_graph_steps(gb_plan *p, int steps)
{
    if (!p) return fail(GB_E_ARG, "null plan");
    if (steps < 0 || steps > kMaxGraphSteps || (steps & 1))
        return fail(GB_E_ARG, "graph steps must be an even number in [0, " + std::to_string(kMaxGraphSteps) + "]");
    p->graph_steps = steps;
    p->release_graph();
    return GB_OK;
}

size_t gb_plan_workspace_bytes(const gb_plan *p, int with_gradient, int checkpoint_every)
{
    if (!p) return 0;
    return layout(p, with_gradient, checkpoint_every).total + 256;
}

size_t gb_plan_gradient_workspace_bytes(const gb_plan *p, int with_rho, int segment_steps, int imaging_format)
{
    if (!p || !img_format_ok(imaging_format)) return 0;
    return layout(p, with_rho ? 2 : 1, segment_steps, imaging_format).total + 256;
}

size_t gb_plan_checkpoint_bytes(const gb_plan *p, int checkpoint_every, int ckpt_format)
{
    if (!p || checkpoint_every < 1 || ckpt_format < GB_CKPT_F32 || ckpt_format > GB_CKPT_F24) return 0;
    const size_t n_ck = (p->d.nt + checkpoint_every - 1) / checkpoint_every;
    return n_ck * ck_bytes(p, ckpt_format);
}

size_t gb_plan_imaging_bytes(const gb_plan *p, int cached_steps, int with_rho, int imaging_format)
{
    if (!p || cached_steps < 0) return 0;
    if (!img_format_ok(imaging_format)) return 0;
    return (size_t)cached_steps * (with_rho ? 3 : 1) * p->d.n_shots * p->plane * img_esize(imaging_format);
}

int gb_forward(gb_plan *P, const float *vp, const float *rho, const float *damp, const float *wavelet,
               float *trace_p, float *trace_vx, float *trace_vz, float *energy_p, float *energy_vx,
               float *energy_vz, int32_t snapshot_every, float *snapshots, const gb_grad_store *store,
               void *workspace, size_t workspace_bytes, void *stream)
{
    g_last_error.clear();
    if (!P || !vp || !rho || !damp || !wavelet) return fail(GB_E_ARG, "null argument");
    if (int rc = check_store(P, store)) return rc;
    const Layout L = layout(P);
    char *ws = aligned_ws(workspace);
    if (!workspace || workspace_bytes < L.total + (size_t)(ws - reinterpret_cast<char *>(workspace)))
        return fail(GB_E_WORKSPACE, "workspace too small");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const gb_model_desc &d = P->d;
    const int S = d.n_shots;
    const bool want_energy = energy_p || energy_vx || energy_vz;
    const int K = store ? std::min<int>(store->checkpoint_every, d.nt) : 0;
    const int t_cache = store ? d.nt - store->cached_steps : d.nt;   // steps >= t_cache keep their imaging fields
    const int n_img = store && store->with_rho ? 3 : 1;

    P->mark(0, true, st);
    Setup Su;
    if (int rc = common_setup(P, L, ws, vp, rho, damp, st, &Su)) return rc;
    float *buf[2] = {reinterpret_cast<float *>(ws + L.fields),
                     reinterpret_cast<float *>(ws + L.fields) + (size_t)S * 3 * P->plane};
    float *energy = reinterpret_cast<float *>(ws + L.energy);
    GB_CUDA(cudaMemsetAsync(buf[0], 0, (size_t)S * 3 * P->plane * 4, st));
    GB_CUDA(cudaMemsetAsync(buf[1], 0, (size_t)S * 3 * P->plane * 4, st));
    if (want_energy) GB_CUDA(cudaMemsetAsync(energy, 0, 3 * P->plane * 4, st));

    if (P->res_tz > 0 && !store && !P->cpml) {
        P->phase_steps[0] += d.nt;
        if (int rc = forward_resident(P, L, ws, Su, buf[0], energy, want_energy, wavelet, trace_p, trace_vx,
                                      trace_vz, snapshot_every, snapshots, st))
            return rc;
        float *eo[3] = {energy_p, energy_vx, energy_vz};
        for (int f = 0; f < 3; ++f)
            if (eo[f]) {
                extract_interior_kernel<<<148, 256, 0, st>>>(energy + f * P->plane, d.nz, d.nx, d.nabc, P->pitch,
                                                             eo[f]);
                GB_CUDA(cudaGetLastError());
                ++P->launches;
            }
        P->mark(0, false, st);
        return GB_OK;
    }
    const StepKernel K0 = fwd_kernel_for(P, want_energy, 0);
    const StepKernel KI = fwd_kernel_for(P, want_energy, n_img == 3 ? 2 : 1);
    if (int rc = prepare_kernel(K0)) return rc;
    if (store && store->cached_steps > 0)
        if (int rc = prepare_kernel(KI)) return rc;
    Maps maps[2];
    for (int b = 0; b < 2; ++b)
        if (int rc = make_maps(P, buf[b], Su.a1, Su.a2, &maps[b])) return rc;

    FwdArgs A{};
    A.g = P->geom();
    A.tile_fast = Su.tile_fast;
    A.a1 = Su.a1; A.k1 = Su.k1; A.a2 = Su.a2; A.k2 = Su.k2; A.k3 = Su.k3;
    A.src_z = Su.d_src; A.src_x = Su.d_src + S;
    A.wavelet = wavelet;
    A.rcv_ptr = Su.d_rptr; A.rcv_ent = Su.d_rent;
    A.tr_p = trace_p; A.tr_vx = trace_vx; A.tr_vz = trace_vz;
    A.energy = want_energy ? energy : nullptr;
    A.img_field_stride = (long long)S * P->plane;
    A.img_fmt = store ? store->imaging_format : GB_IMG_F32;
    A.err = Su.err;
    A.cpml = Su.cpml;
    const size_t img_es = store ? img_esize(store->imaging_format) : 4;

    GroupStreams gs;
    if (int rc = group_streams(P, st, &gs)) return rc;
    if (int rc = fork(gs)) return rc;
    const size_t step_img = (size_t)n_img * S * P->plane;
    int snap_i = 0;
    P->phase_steps[0] += d.nt;
    int it_first = 0;
    // plain forward: whole chunks of graph_steps steps as graph replays
    const int C = P->graph_steps;
    const bool snaps_fit = snapshot_every <= 0 || !snapshots || snapshot_every % std::max(C, 1) == 0;
    if (C > 0 && !store && snaps_fit && d.nt >= C) {
        if (int rc = join(gs)) return rc;            // the chunks run from the caller's stream
        int *step_ctr = reinterpret_cast<int *>(ws + L.err + 128);
        int dev = -1;
        GB_CUDA(cudaGetDevice(&dev));
        const std::vector<uintptr_t> key = {
            (uintptr_t)dev, (uintptr_t)ws, (uintptr_t)wavelet, (uintptr_t)trace_p, (uintptr_t)trace_vx,
            (uintptr_t)trace_vz, (uintptr_t)want_energy, (uintptr_t)C, (uintptr_t)P->tz, (uintptr_t)P->spc_eff,
            (uintptr_t)P->n_groups, (uintptr_t)gs.n, (uintptr_t)K0.fn, (uintptr_t)P->sched};
        if (!P->gexec || P->gkey != key) {
            P->release_graph();
            if (int rc = capture_forward_chunk(P, K0, maps, buf, Su.psi, A, C, step_ctr, &P->gexec)) return rc;
            P->gkey = key;
        }
        step_set_kernel<<<1, 1, 0, st>>>(step_ctr, 0);
        GB_CUDA(cudaGetLastError());
        ++P->launches;
        const int n_chunks = d.nt / C;
        for (int k = 0; k < n_chunks; ++k) {
            GB_CUDA(cudaGraphLaunch(P->gexec, st));
            P->launches += (long long)C * gs.n + 1;
            ++P->api_launches;
            const int last = (k + 1) * C - 1;
            if (snapshot_every > 0 && snapshots && ((last + 1) % snapshot_every == 0 || last == d.nt - 1)) {
                GB_CUDA(cudaMemcpy2DAsync(snapshots + (size_t)snap_i * d.nz * d.nx, (size_t)d.nx * 4,
                                          buf[0] + (size_t)d.nabc * P->pitch + d.nabc, (size_t)P->pitch * 4,
                                          (size_t)d.nx * 4, d.nz, cudaMemcpyDeviceToDevice, st));
                ++snap_i;
            }
        }
        it_first = n_chunks * C;
        if (int rc = fork(gs)) return rc;
    }
    auto one_step = [&](int it) -> int {
        const int b = it & 1;
        A.it = it;
        A.out = buf[b ^ 1];
        if (Su.cpml) {
            A.psi_in = Su.psi[b];
            A.psi_out = Su.psi[b ^ 1];
        }
        const bool keep = store && it >= t_cache;
        A.imaging = keep ? img_at(store->imaging, (size_t)(it - t_cache) * step_img, img_es) : nullptr;
        for (int i = 0; i < gs.n; ++i) {
            int g0, gc;
            launch_groups(gs, i, P->n_groups, &g0, &gc);
            const cudaStream_t si = gs.at(i);
            if (store && it < t_cache && it % K == 0) {
                const int s0 = P->group_first(g0);
                const int ns = gs.n == 1 ? S : P->group_shots(g0);
                if (int rc = save_checkpoint(P, buf[b], store->checkpoints, it / K, store->format, Su.amax, s0, ns, si))
                    return rc;
            }
            if (int rc = launch_step(P, keep ? KI : K0, maps[b], A, g0, gc, si)) return rc;
            if (snapshot_every > 0 && snapshots && g0 == 0 && ((it + 1) % snapshot_every == 0 || it == d.nt - 1)) {
                GB_CUDA(cudaMemcpy2DAsync(snapshots + (size_t)snap_i * d.nz * d.nx, (size_t)d.nx * 4,
                                          buf[b ^ 1] + (size_t)d.nabc * P->pitch + d.nabc, (size_t)P->pitch * 4,
                                          (size_t)d.nx * 4, d.nz, cudaMemcpyDeviceToDevice, si));
                ++snap_i;
            }
        }
        return GB_OK;
    };
    int it = it_first;
    // the steps that keep their imaging fields (a gradient's forward): chunks
    // of C steps replayed from one CUDA graph, from an even step on (the
    // state level of step j of a chunk is j & 1); the imaging fields' address
    // comes from the device step counter
    if (store && C > 0 && (snapshot_every <= 0 || !snapshots) && !P->stream_usable() && d.nt - t_cache >= C) {
        for (; it < d.nt && (it < t_cache || (it & 1)); ++it)
            if (int rc = one_step(it)) return rc;
        if (d.nt - it >= C) {
            if (int rc = join(gs)) return rc;
            int *step_ctr = reinterpret_cast<int *>(ws + L.err + 128);
            int dev = -1;
            GB_CUDA(cudaGetDevice(&dev));
            const std::vector<uintptr_t> key = {
                (uintptr_t)dev, (uintptr_t)ws, (uintptr_t)wavelet, (uintptr_t)trace_p, (uintptr_t)trace_vx,
                (uintptr_t)trace_vz, (uintptr_t)want_energy, (uintptr_t)C, (uintptr_t)P->tz, (uintptr_t)P->spc_eff,
                (uintptr_t)P->n_groups, (uintptr_t)gs.n, (uintptr_t)KI.fn, (uintptr_t)store->imaging,
                (uintptr_t)t_cache, (uintptr_t)store->imaging_format, (uintptr_t)store->with_rho, (uintptr_t)P->sched};
            FwdArgs B = A;
            B.step_base = step_ctr;
            B.img_base = reinterpret_cast<float *>(store->imaging);
            B.img_step = (long long)step_img;
            B.img_t0 = t_cache;
            B.imaging = reinterpret_cast<float *>(store->imaging);
            if (int rc = capture_chunk(P, P->g_fwd_img, key, C, step_ctr, C, true, [&](int j, const GroupStreams &g) {
                    FwdArgs Bj = B;
                    Bj.it = j;
                    Bj.out = buf[(j & 1) ^ 1];
                    if (Su.cpml) {
                        Bj.psi_in = Su.psi[j & 1];
                        Bj.psi_out = Su.psi[(j & 1) ^ 1];
                    }
                    for (int i = 0; i < g.n; ++i) {
                        int g0, gc;
                        launch_groups(g, i, P->n_groups, &g0, &gc);
                        if (int rc = launch_step(P, KI, maps[j & 1], Bj, g0, gc, g.at(i))) return rc;
                    }
                    return GB_OK;
                }))
                return rc;
            step_set_kernel<<<1, 1, 0, st>>>(step_ctr, it);
            GB_CUDA(cudaGetLastError());
            ++P->launches;
            ++P->api_launches;
            for (; d.nt - it >= C; it += C) {
                GB_CUDA(cudaGraphLaunch(P->g_fwd_img.exec, st));
                P->launches += (long long)C * gs.n + 1;
                ++P->api_launches;
            }
            if (int rc = fork(gs)) return rc;
        }
    }
    for (; it < d.nt; ++it)
        if (int rc = one_step(it)) return rc;
    if (int rc = join(gs)) return rc;
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

int gb_trace_misfit(const float *pred, const float *obs, int32_t n_shots, int32_t nt, int32_t n_rcv, float *adj,
                    float *per_trace, float *loss, void *stream)
{
    g_last_error.clear();
    if (!pred || !obs || !per_trace || !loss) return fail(GB_E_ARG, "null argument");
    if (n_shots < 1 || nt < 1 || n_rcv < 1) return fail(GB_E_ARG, "n_shots, nt and n_rcv must be >= 1");
    if (n_shots > 65535) return fail(GB_E_ARG, "at most 65535 shots per call");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    dim3 grid((n_rcv + 127) / 128, n_shots);
    trace_misfit_kernel<<<grid, 128, 0, st>>>(pred, obs, nt, n_rcv, adj, per_trace);
    GB_CUDA(cudaGetLastError());
    trace_misfit_sum_kernel<<<1, 1024, 0, st>>>(per_trace, (long long)n_shots * n_rcv, loss);
    GB_CUDA(cudaGetLastError());
    return GB_OK;
}

size_t gb_plan_autotune_workspace_bytes(gb_plan *p)
{
    if (!p) return 0;
    const int tz = p->tz, rm = p->res_mode, rt = p->res_tz_req;
    size_t m = 0;
    for (int t : {16, 32}) {
        p->tz = t;
        p->res_mode = 0;
        p->retile();
        m = std::max(m, gb_plan_workspace_bytes(p, 0, 0));
    }
    for (int mode : {1, 3}) {
        p->res_mode = mode;
        for (int t : kResidentRows) {
            p->res_tz_req = t;
            p->res_choose();
            m = std::max(m, gb_plan_workspace_bytes(p, 0, 0));
        }
    }
    p->tz = tz;
    p->res_mode = rm;
    p->res_tz_req = rt;
    p->retile();
    return m;
}

int gb_plan_autotune(gb_plan *P, const float *vp, const float *rho, const float *damp, const float *wavelet,
                     void *workspace, size_t workspace_bytes, int32_t steps, void *stream, float *best_ms_per_step)
{
    g_last_error.clear();
    if (!P || !vp || !rho || !damp || !wavelet || !workspace) return fail(GB_E_ARG, "null argument");
    if (steps < 2 || steps > P->d.nt) return fail(GB_E_ARG, "steps must be in [2, nt]");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    struct Config {
        int tz, spc;
        bool streams;
        int graph;
        bool stream;
        int res;    // resident forward tile rows, 0 = the tile kernel
        int xm;     // its gb_plan_set_resident mode (1 global, 2 cluster, 3 one exchange a step)
    };
    const Config saved{P->tz, P->spc, P->group_streams, P->graph_steps, P->stream, P->res_tz,
                       P->res_exchange() == 1 ? 2 : P->res_exchange() == 2 ? 3 : 1};
    const int saved_res_mode = P->res_mode, saved_res_req = P->res_tz_req;
    const bool prof = P->prof;
    const int nt = P->d.nt;
    const long long launches = P->launches;
    const int S = P->d.n_shots;
    const int C = 16;
    const int n = steps >= C ? steps / C * C : steps;       // whole graph chunks when graphs are tried
    std::vector<Config> cands;
    for (int stream = 0; stream <= (P->d.free_surface ? 0 : 1); ++stream)
        for (int tz : {16, 32}) {
            if (stream && tz != 16) continue;      // the streaming kernel walks 16-row chunks
            for (int spc : {0, 1, 2, 4, 8, 16}) {
                if (spc > S) continue;
                for (int streams = 1; streams >= 0; --streams)
                    for (int graph : {0, C}) {
                        if (graph > n) continue;
                        cands.push_back({tz, spc, streams != 0, graph, stream != 0, 0, 0});
                    }
            }
        }
    if (!P->cpml)
        for (int tz : kResidentRows)
            if (P->res_fits(tz, gb_plan::sm_count())) {
                cands.push_back({saved.tz, saved.spc, true, 0, false, tz, 1});
                if (P->res_single_ok()) cands.push_back({saved.tz, saved.spc, true, 0, false, tz, 3});
                const long long n = (long long)((P->Nx + TX - 1) / TX) * ((P->Nz + tz - 1) / tz);
                if (n <= gb_plan::kMaxClusterTiles) cands.push_back({saved.tz, saved.spc, true, 0, false, tz, 2});
            }
    cudaEvent_t e0, e1;
    GB_CUDA(cudaEventCreate(&e0));
    GB_CUDA(cudaEventCreate(&e1));
    P->prof = false;
    P->d.nt = n;                       // time n steps; the wavelet is read within its first S * n samples
    float best = -1.f;
    Config win = saved;
    int rc = GB_OK;
    for (const Config &k : cands) {
        P->tz = k.tz;
        P->spc = k.spc;
        P->retile();
        P->group_streams = k.streams;
        P->graph_steps = k.graph;
        P->stream = k.stream;
        P->res_mode = k.res ? k.xm : 0;
        P->res_tz_req = k.res;
        P->res_choose();
        P->release_graph();
        if (k.res && P->res_tz != k.res) continue;
        if (gb_plan_workspace_bytes(P, 0, 0) > workspace_bytes) continue;
        if (!k.res && k.streams && P->n_groups == 1) continue;      // same as without
        float ms = -1.f;
        for (int rep = 0; rep < 3 && rc == GB_OK; ++rep) {
            if (cudaEventRecord(e0, st) != cudaSuccess) rc = fail(GB_E_CUDA, "event record failed");
            if (rc == GB_OK)
                rc = gb_forward(P, vp, rho, damp, wavelet, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0,
                                nullptr, nullptr, workspace, workspace_bytes, stream);
            if (rc == GB_OK && (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess))
                rc = fail(GB_E_CUDA, "event wait failed");
            float t = 0.f;
            if (rc == GB_OK && rep > 0 && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess)
                ms = ms < 0 ? t : std::min(ms, t);   // the first run warms up (and captures a graph)
        }
        if (rc != GB_OK) break;
        if (ms >= 0 && (best < 0 || ms < best)) {
            best = ms;
            win = k;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    P->d.nt = nt;
    P->prof = prof;
    P->launches = launches;
    P->tz = win.tz;
    P->spc = win.spc;
    P->retile();
    P->group_streams = win.streams;
    P->graph_steps = win.graph;
    P->stream = win.stream;
    if (best < 0) {
        P->res_mode = saved_res_mode;
        P->res_tz_req = saved_res_req;
    } else {
        P->res_mode = win.res ? win.xm : 0;
        P->res_tz_req = win.res;
    }
    P->res_choose();
    P->release_graph();                // captured with the shortened step count
    if (rc != GB_OK) return rc;
    if (best < 0) return fail(GB_E_WORKSPACE, "no candidate fits the workspace");
    if (best_ms_per_step) *best_ms_per_step = best / n;
    return GB_OK;
}

int gb_backward(gb_plan *P, const float *vp, const float *rho, const float *damp, const float *wavelet,
                const float *res_p, const float *res_vx, const float *res_vz, const gb_grad_store *store,
                float *grad_vp, float *grad_rho, float *grad_wavelet, void *workspace, size_t workspace_bytes,
                void *stream)
{
    g_last_error.clear();
    if (!P || !vp || !rho || !damp || !wavelet || !store || !grad_vp) return fail(GB_E_ARG, "null argument");
    if (int rc = check_store(P, store)) return rc;
    if (grad_rho && !store->with_rho) return fail(GB_E_ARG, "density gradient needs a store made with with_rho");
    if (grad_wavelet) {
        // the adjoint keeps lambda_p on the p mask only (cells off it never
        // depend on the model); a source off it would need the dropped part
        const StepGeom gm = P->geom();
        for (int s = 0; s < P->d.n_shots; ++s)
            if (P->src_z[s] < gm.p_r0 || P->src_z[s] > gm.p_r1 || P->src_x[s] < gm.p_c0 || P->src_x[s] > gm.p_c1)
                return fail(GB_E_UNSUPPORTED, "wavelet gradients need every source inside the p update region");
        GB_CUDA(cudaMemsetAsync(grad_wavelet, 0, (size_t)P->d.n_shots * P->d.nt * 4,
                                reinterpret_cast<cudaStream_t>(stream)));
    }
    if (P->cpml)
        return backward_cpml(P, vp, rho, damp, res_p, res_vx, res_vz, store, grad_vp, grad_rho, grad_wavelet,
                             workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream));
    const gb_model_desc &d = P->d;
    const int S = d.n_shots;
    const int K = std::min<int>(store->checkpoint_every, d.nt);
    const bool rho_fields = store->with_rho != 0;
    const int with_grad = rho_fields ? 2 : 1;
    // recompute segments lie in [0, nt - cached_steps): the segment buffer
    // holds at most that many steps
    const int ifmt = store->imaging_format;
    const Layout L = layout(P, with_grad, std::max(1, std::min(K, d.nt - store->cached_steps)), ifmt);
    char *ws = aligned_ws(workspace);
    if (!workspace || workspace_bytes < L.total + (size_t)(ws - reinterpret_cast<char *>(workspace)))
        return fail(GB_E_WORKSPACE, "workspace too small");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

    Setup Su;
    if (int rc = common_setup(P, L, ws, vp, rho, damp, st, &Su)) return rc;
    const size_t state_fl = (size_t)S * 3 * P->plane;
    float *fb[2] = {reinterpret_cast<float *>(ws + L.fields), reinterpret_cast<float *>(ws + L.fields) + state_fl};
    float *mu[2] = {reinterpret_cast<float *>(ws + L.mu), reinterpret_cast<float *>(ws + L.mu) + state_fl};
    void *wimg = ws + L.img;      // imaging fields of one recompute segment, in the store's format
    float *G1 = reinterpret_cast<float *>(ws + L.g1), *C1 = reinterpret_cast<float *>(ws + L.c1);
    float *G2 = rho_fields ? reinterpret_cast<float *>(ws + L.g2) : nullptr;
    float *C2 = rho_fields ? reinterpret_cast<float *>(ws + L.c2) : nullptr;
    int *d_aptr = reinterpret_cast<int *>(ws + L.arcv_ptr);
    int4 *d_aent = reinterpret_cast<int4 *>(ws + L.arcv_ent);
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

    const bool fs = d.free_surface != 0;
    const StepKernel KF = fwd_kernel_for(P, false, rho_fields ? 2 : 1);
    // cached and recomputed imaging fields share the store's format
    const StepKernel KA = adj_kernel(P->R, P->tz, fs, rho_fields, ifmt);
    if (int rc = prepare_kernel(KF)) return rc;
    if (int rc = prepare_kernel(KA)) return rc;
    Maps fmaps[2], amaps[2];
    for (int b = 0; b < 2; ++b) {
        if (int rc = make_maps(P, fb[b], Su.a1, Su.a2, &fmaps[b])) return rc;
        if (int rc = make_maps(P, mu[b], Su.a1, Su.a2, &amaps[b])) return rc;
    }

    const StepGeom g = P->geom();
    FwdArgs F{};
    F.g = g;
    F.a1 = Su.a1; F.k1 = Su.k1; F.a2 = Su.a2; F.k2 = Su.k2; F.k3 = Su.k3;
    F.tile_fast = Su.tile_fast;
    F.src_z = Su.d_src; F.src_x = Su.d_src + S;
    F.wavelet = wavelet;
    F.rcv_ptr = Su.d_rptr; F.rcv_ent = Su.d_rent;
    F.err = Su.err;
    F.img_field_stride = (long long)S * P->plane;
    F.img_fmt = ifmt;
    AdjArgs A{};
    A.g = g;
    A.a1 = Su.a1; A.k1 = Su.k1; A.a2 = Su.a2; A.k2 = Su.k2; A.k3 = Su.k3;
    A.tile_fast = Su.tile_fast;
    A.rcv_ptr = d_aptr; A.rcv_ent = d_aent;
    A.res_p = res_p; A.res_vx = res_vx; A.res_vz = res_vz;
    A.img_field_stride = (long long)S * P->plane;
    A.G1 = G1; A.C1 = C1; A.G2 = G2; A.C2 = C2;
    A.err = Su.err;
    A.grad_wavelet = grad_wavelet;
    A.src_z = Su.d_src;
    A.src_x = Su.d_src + S;

    GroupStreams gs;
    if (int rc = group_streams(P, st, &gs)) return rc;
    const size_t step_img = (size_t)(rho_fields ? 3 : 1) * S * P->plane;
    const int t_cache = d.nt - store->cached_steps;
    int cur = 0;   // adjoint state lives in mu[cur]

    // adjoint sweep over [t0, t1) in reverse, imaging fields at img_base[(it - t0)]
    const int C = P->graph_steps;
    int *step_ctr = reinterpret_cast<int *>(ws + L.err + 128);
    // with `graph`, chunks of C steps that start on adjoint level 0 are
    // replayed from one CUDA graph (the step index and the imaging fields'
    // address come from a device counter counting down)
    auto adjoint_sweep = [&](int t0, int t1, void *img_base, int img_fmt, bool graph) -> int {
        P->mark(2, true, st);
        P->phase_steps[2] += t1 - t0;
        if (int rc = fork(gs)) return rc;
        auto one_step = [&](int it) -> int {
            A.it = it;
            A.out = mu[cur ^ 1];
            A.img = img_at(img_base, (size_t)(it - t0) * step_img, img_esize(img_fmt));
            A.img_fmt = img_fmt;
            for (int i = 0; i < gs.n; ++i) {
                int g0, gc;
                launch_groups(gs, i, P->n_groups, &g0, &gc);
                if (int rc = launch_step(P, KA, amaps[cur], A, g0, gc, gs.at(i))) return rc;
            }
            cur ^= 1;
            return GB_OK;
        };
        int it = t1 - 1;
        if (graph && C > 0 && t1 - t0 >= C) {
            for (; it >= t0 && cur != 0; --it)
                if (int rc = one_step(it)) return rc;
            if (it - t0 + 1 >= C) {
                if (int rc = join(gs)) return rc;
                int dev = -1;
                GB_CUDA(cudaGetDevice(&dev));
                const std::vector<uintptr_t> key = {
                    (uintptr_t)dev, (uintptr_t)ws, (uintptr_t)res_p, (uintptr_t)res_vx, (uintptr_t)res_vz,
                    (uintptr_t)img_base, (uintptr_t)img_fmt, (uintptr_t)t0, (uintptr_t)grad_wavelet, (uintptr_t)C,
                    (uintptr_t)P->tz, (uintptr_t)P->spc_eff, (uintptr_t)P->n_groups, (uintptr_t)gs.n,
                    (uintptr_t)KA.fn, (uintptr_t)rho_fields, (uintptr_t)P->sched};
                AdjArgs B = A;
                B.step_base = step_ctr;
                B.img_base = reinterpret_cast<float *>(img_base);
                B.img_step = (long long)step_img;
                B.img_t0 = t0;
                B.img_fmt = img_fmt;
                if (int rc = capture_chunk(P, P->g_adj, key, C, step_ctr, -C, true, [&](int j, const GroupStreams &g) {
                        AdjArgs Bj = B;
                        Bj.it = j;
                        Bj.out = mu[(j & 1) ^ 1];
                        for (int i = 0; i < g.n; ++i) {
                            int g0, gc;
                            launch_groups(g, i, P->n_groups, &g0, &gc);
                            if (int rc = launch_step(P, KA, amaps[j & 1], Bj, g0, gc, g.at(i))) return rc;
                        }
                        return GB_OK;
                    }))
                    return rc;
                step_set_kernel<<<1, 1, 0, st>>>(step_ctr, it);
                GB_CUDA(cudaGetLastError());
                ++P->launches;
                ++P->api_launches;
                for (; it - t0 + 1 >= C; it -= C) {
                    GB_CUDA(cudaGraphLaunch(P->g_adj.exec, st));
                    P->launches += (long long)C * gs.n + 1;
                    ++P->api_launches;
                }
                if (int rc = fork(gs)) return rc;
            }
        }
        for (; it >= t0; --it)
            if (int rc = one_step(it)) return rc;
        if (int rc = join(gs)) return rc;
        P->mark(2, false, st);
        return GB_OK;
    };

    // 1. steps whose imaging fields the forward kept
    if (store->cached_steps > 0)
        if (int rc = adjoint_sweep(t_cache, d.nt, store->imaging, store->imaging_format, true)) return rc;
    // 2. earlier steps, one checkpoint segment at a time: fp32 recompute from
    //    the checkpoint (writing the imaging fields), then the adjoint sweep
    const int n_seg = (t_cache + K - 1) / K;
    for (int seg = n_seg - 1; seg >= 0; --seg) {
        const int t0 = seg * K, t1 = std::min(t_cache, t0 + K);
        P->mark(1, true, st);
        P->phase_steps[1] += t1 - t0;
        if (int rc = fork(gs)) return rc;
        for (int i = 0; i < gs.n; ++i) {
            int g0, gc;
            launch_groups(gs, i, P->n_groups, &g0, &gc);
            const int s0 = P->group_first(g0), ns = gs.n == 1 ? S : P->group_shots(g0);
            if (int rc = restore_checkpoint(P, fb[0], store->checkpoints, seg, store->format, s0, ns, gs.at(i)))
                return rc;
        }
        for (int it = t0; it < t1; ++it) {
            const int b = (it - t0) & 1;
            F.it = it;
            F.out = fb[b ^ 1];
            F.imaging = img_at(wimg, (size_t)(it - t0) * step_img, img_esize(ifmt));
            for (int i = 0; i < gs.n; ++i) {
                int g0, gc;
                launch_groups(gs, i, P->n_groups, &g0, &gc);
                if (int rc = launch_step(P, KF, fmaps[b], F, g0, gc, gs.at(i))) return rc;
            }
        }
        if (int rc = join(gs)) return rc;
        P->mark(1, false, st);
        if (int rc = adjoint_sweep(t0, t1, wimg, ifmt, false)) return rc;
    }
    grad_finish_kernel<<<4 * 148, 256, 0, st>>>(vp, rho, G1, C1, G2, C2, P->n_groups, P->plane, d.nz, d.nx, d.nabc,
                                                P->pitch, grad_vp, grad_rho);
    GB_CUDA(cudaGetLastError());
    ++P->launches;
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

int gb_selftest_bounded_wait(void *workspace, size_t workspace_bytes, int32_t complete, int32_t max_polls,
                             void *stream)
{
    g_last_error.clear();
    if (!workspace) return fail(GB_E_ARG, "null workspace");
    char *ws = reinterpret_cast<char *>(align256(reinterpret_cast<uintptr_t>(workspace)));
    if (ws + 4 > reinterpret_cast<char *>(workspace) + workspace_bytes) return fail(GB_E_WORKSPACE, "workspace too small");
    if (max_polls < 1 || (uint32_t)max_polls > kMaxPolls) return fail(GB_E_ARG, "max_polls out of [1, 2^22]");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    GB_CUDA(cudaMemsetAsync(ws, 0, 4, st));
    bounded_wait_selftest_kernel<<<1, 64, 0, st>>>(reinterpret_cast<int *>(ws), complete != 0, (uint32_t)max_polls);
    GB_CUDA(cudaGetLastError());
    return gb_workspace_status(workspace, stream);
}

int gb_plan_launch_calls(const gb_plan *P, long long *calls)
{
    if (!P || !calls) return fail(GB_E_ARG, "null argument");
    *calls = P->api_launches;
    return GB_OK;
}

int gb_plan_set_profiling(gb_plan *P, int enable)
{
    if (!P) return fail(GB_E_ARG, "null plan");
    P->prof = enable != 0;
    P->clear_events();
    P->launches = 0;
    P->api_launches = 0;
    for (auto &n : P->phase_steps) n = 0;
    return GB_OK;
}

int gb_plan_profile(gb_plan *P, double *ms_forward, double *ms_recompute, double *ms_adjoint, long long *launches,
                    long long *phase_steps)
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
    if (phase_steps)
        for (int ph = 0; ph < 3; ++ph) phase_steps[ph] = P->phase_steps[ph];
    P->clear_events();
    P->launches = 0;
    for (auto &n : P->phase_steps) n = 0;
    return GB_OK;
}

}  // extern "C"


// ---------------------------------------------------------------------------
// Batches of models: one launch per time step for all of them.
// ---------------------------------------------------------------------------
namespace {

struct BatchLayout {
    size_t models, maps, items, clock, total;
    long long n_items;
};

BatchLayout batch_layout(gb_plan *const *plans, int n)
{
    BatchLayout B{};
    B.n_items = 0;
    for (int m = 0; m < n; ++m) B.n_items += (long long)plans[m]->n_tiles * plans[m]->n_groups;
    size_t o = 0;
    B.models = o; o = align256(o + (size_t)n * sizeof(BatchModel));
    B.maps = o; o = align256(o + (size_t)n * sizeof(BatchMaps));
    B.items = o; o = align256(o + (size_t)std::max<long long>(B.n_items, 1) * 16);
    B.clock = o; o = align256(o + 4);            // step counter of graph-replayed chunks
    B.total = o;
    return B;
}

int check_batch(gb_plan *const *plans, int n, const gb_model_io *io, bool gradient)
{
    if (!plans || !io || n < 1) return fail(GB_E_ARG, "empty batch");
    for (int m = 0; m < n; ++m) {
        const gb_plan *P = plans[m];
        if (!P) return fail(GB_E_ARG, "null plan in batch");
        if (P->R != plans[0]->R || (P->d.free_surface != 0) != (plans[0]->d.free_surface != 0))
            return fail(GB_E_ARG, "a batch needs one stencil order and one free-surface setting");
        if (P->tz != 16) return fail(GB_E_ARG, "batched plans use 16-row tiles (gb_plan_set_tiling(plan, 16, ...))");
        if (P->cpml) return fail(GB_E_UNSUPPORTED, "batched runs use the damping layers, not CPML");
        const gb_model_io &x = io[m];
        if (!x.vp || !x.rho || !x.damp || !x.wavelet || !x.workspace) return fail(GB_E_ARG, "null model input");
        if (gradient) {
            if (!x.store || !x.grad_vp) return fail(GB_E_ARG, "gradient needs a store and grad_vp for every model");
            if (int rc = check_store(P, x.store)) return rc;
            if (x.store->checkpoint_every != io[0].store->checkpoint_every ||
                (x.store->with_rho != 0) != (io[0].store->with_rho != 0) || x.store->format != io[0].store->format)
                return fail(GB_E_ARG, "a batch shares checkpoint_every, format and with_rho");
            if (x.grad_rho && !x.store->with_rho) return fail(GB_E_ARG, "density gradient needs with_rho stores");
        } else if (x.store) {
            if (int rc = check_store(P, x.store)) return rc;
            if (x.store->checkpoint_every != io[0].store->checkpoint_every ||
                (x.store->with_rho != 0) != (io[0].store->with_rho != 0))
                return fail(GB_E_ARG, "a batch shares checkpoint_every and with_rho");
        }
    }
    return GB_OK;
}

int upload_batch(gb_plan *const *plans, int n, const std::vector<BatchModel> &models,
                 const std::vector<BatchMaps> &maps, char *bws, const BatchLayout &B, cudaStream_t st)
{
    std::vector<int4> items;
    items.reserve(B.n_items);
    for (int m = 0; m < n; ++m)
        for (int t = 0; t < plans[m]->n_tiles; ++t)
            for (int g = 0; g < plans[m]->n_groups; ++g) items.push_back(int4{m, t, g, 0});
    GB_CUDA(cudaMemcpyAsync(bws + B.models, models.data(), n * sizeof(BatchModel), cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemcpyAsync(bws + B.maps, maps.data(), n * sizeof(BatchMaps), cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemcpyAsync(bws + B.items, items.data(), items.size() * 16, cudaMemcpyHostToDevice, st));
    return GB_OK;
}

int make_state_maps(const gb_plan *P, const float *buf, CUtensorMap (&m)[3])
{
    const int n_planes = 3 * P->d.n_shots;
    if (int rc = make_map(&m[0], buf, P->Nx, P->Nz, P->pitch, n_planes, RW, box_rows_p(P->R, P->tz))) return rc;
    if (int rc = make_map(&m[1], buf, P->Nx, P->Nz, P->pitch, n_planes, VXW, box_rows_p(P->R, P->tz))) return rc;
    return make_map(&m[2], buf, P->Nx, P->Nz, P->pitch, n_planes, RW, box_rows_vz(P->R, P->tz));
}

int launch_batch(gb_plan *P0, const StepKernel &K, long long n_items, void **args, cudaStream_t st)
{
    GB_CUDA(cudaLaunchKernel(K.fn, dim3((unsigned)n_items), dim3(NTHR), args, K.smem, st));
    ++P0->launches;
    ++P0->api_launches;
    return GB_OK;
}

// The lanes of a batch: its models split into up to kBatchLanes runs of
// consecutive models with about equal work items.  Inside a step graph each
// lane's launches go to a stream of their own, so a lane starts its next
// step while the others finish this one (no model depends on another).
constexpr int kBatchLanes = 4;
struct BatchLanes {
    int n = 1;
    long long off[kBatchLanes] = {0}, cnt[kBatchLanes] = {0};
};

BatchLanes batch_lanes(gb_plan *const *plans, int n_models, long long n_items)
{
    BatchLanes L;
    const int want = std::min(kBatchLanes, n_models);
    L.cnt[0] = n_items;
    if (want < 2) return L;
    long long acc = 0;
    int lane = 0;
    L.off[0] = 0;
    for (int m = 0; m < n_models; ++m) {
        const long long w = (long long)plans[m]->n_tiles * plans[m]->n_groups;
        // close the lane once it holds its share (keeping a model for each later lane)
        if (lane + 1 < want && acc > 0 && acc + w / 2 > n_items * (lane + 1) / want &&
            n_models - m >= want - lane - 1) {
            L.cnt[lane] = acc - L.off[lane];
            L.off[++lane] = acc;
        }
        acc += w;
    }
    L.cnt[lane] = acc - L.off[lane];
    L.n = lane + 1;
    return L;
}

// A batched step loop in chunks of C steps replayed from the CUDA graph in
// `slot` (captured once per key): launch(j, lane, stream) launches step j of
// a chunk for one lane, the kernels reading the batch clock at `clock`,
// which starts at `first` and moves by `dir` * C after each chunk.
template <class Launch>
int batch_graph_chunks(gb_plan *P0, gb_plan::GraphSlot &slot, const std::vector<uintptr_t> &key, int C, int *clock,
                       int first, int dir, int n_chunks, const BatchLanes &lanes, cudaStream_t st, Launch launch)
{
    if (int rc = capture_chunk(
            P0, slot, key, C, clock, dir * C, lanes.n > 1,
            [&](int j, const GroupStreams &g) {
                for (int i = 0; i < lanes.n; ++i)
                    if (int rc = launch(j, i, lanes.n > 1 ? g.at(i) : g.main)) return rc;
                return (int)GB_OK;
            },
            lanes.n))
        return rc;
    step_set_kernel<<<1, 1, 0, st>>>(clock, first);
    GB_CUDA(cudaGetLastError());
    ++P0->launches;
    ++P0->api_launches;
    for (int k = 0; k < n_chunks; ++k) {
        GB_CUDA(cudaGraphLaunch(slot.exec, st));
        P0->launches += (long long)C * lanes.n + 1;
        ++P0->api_launches;
    }
    return GB_OK;
}

}  // namespace

extern "C" {

size_t gb_batch_workspace_bytes(gb_plan *const *plans, int n_models)
{
    if (!plans || n_models < 1) return 0;
    for (int m = 0; m < n_models; ++m)
        if (!plans[m]) return 0;
    return batch_layout(plans, n_models).total + 256;
}

int gb_batch_forward(gb_plan *const *plans, int n, const gb_model_io *io, void *batch_workspace,
                     size_t batch_workspace_bytes, void *stream)
{
    g_last_error.clear();
    if (int rc = check_batch(plans, n, io, false)) return rc;
    const BatchLayout B = batch_layout(plans, n);
    char *bws = aligned_ws(batch_workspace);
    if (!batch_workspace || batch_workspace_bytes < B.total + (size_t)(bws - reinterpret_cast<char *>(batch_workspace)))
        return fail(GB_E_WORKSPACE, "batch workspace too small");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    gb_plan *P0 = plans[0];
    const bool fs = P0->d.free_surface != 0;
    std::vector<BatchModel> models(n);
    std::vector<BatchMaps> maps(n);
    bool any_energy = false, any_cache = false, rho = false;
    int maxnt = 0;
    P0->mark(0, true, st);
    for (int m = 0; m < n; ++m) {
        gb_plan *P = plans[m];
        const gb_model_io &x = io[m];
        const Layout L = layout(P);
        char *ws = aligned_ws(x.workspace);
        if (x.workspace_bytes < L.total + (size_t)(ws - reinterpret_cast<char *>(x.workspace)))
            return fail(GB_E_WORKSPACE, "workspace of model " + std::to_string(m) + " too small");
        Setup Su;
        if (int rc = common_setup(P, L, ws, x.vp, x.rho, x.damp, st, &Su)) return rc;
        const int S = P->d.n_shots;
        float *buf0 = reinterpret_cast<float *>(ws + L.fields), *buf1 = buf0 + (size_t)S * 3 * P->plane;
        float *energy = reinterpret_cast<float *>(ws + L.energy);
        const bool want_energy = x.energy_p || x.energy_vx || x.energy_vz;
        GB_CUDA(cudaMemsetAsync(buf0, 0, (size_t)2 * S * 3 * P->plane * 4, st));
        if (want_energy) GB_CUDA(cudaMemsetAsync(energy, 0, 3 * P->plane * 4, st));
        BatchModel &M = models[m];
        M = BatchModel{};
        FwdArgs &F = M.f;
        F.g = P->geom();
        F.a1 = Su.a1; F.k1 = Su.k1; F.a2 = Su.a2; F.k2 = Su.k2; F.k3 = Su.k3;
        F.tile_fast = Su.tile_fast;
        F.src_z = Su.d_src; F.src_x = Su.d_src + S;
        F.wavelet = x.wavelet;
        F.rcv_ptr = Su.d_rptr; F.rcv_ent = Su.d_rent;
        F.tr_p = x.trace_p; F.tr_vx = x.trace_vx; F.tr_vz = x.trace_vz;
        F.energy = want_energy ? energy : nullptr;
        F.img_field_stride = (long long)S * P->plane;
        F.err = Su.err;
        M.fld[0] = buf0;
        M.fld[1] = buf1;
        M.nt = P->d.nt;
        const gb_grad_store *sto = x.store;
        M.K = sto ? std::min<int>(sto->checkpoint_every, P->d.nt) : P->d.nt;
        M.t_cache = sto ? P->d.nt - sto->cached_steps : P->d.nt;
        M.cache = sto && sto->cached_steps > 0 ? reinterpret_cast<float *>(sto->imaging) : nullptr;
        M.cache_fmt = sto ? sto->imaging_format : GB_IMG_F32;
        M.step_img = (long long)((sto && sto->with_rho) ? 3 : 1) * S * P->plane;
        if (int rc = make_state_maps(P, buf0, maps[m].fld[0])) return rc;
        if (int rc = make_state_maps(P, buf1, maps[m].fld[1])) return rc;
        if (int rc = make_map2d(&maps[m].a1, Su.a1, P->Nx, P->Nz, P->pitch, RW, box_rows_p(P->R, P->tz))) return rc;
        if (int rc = make_map2d(&maps[m].a2, Su.a2, P->Nx, P->Nz, P->pitch, RW, P->tz)) return rc;
        any_energy |= want_energy;
        any_cache |= M.cache != nullptr;
        rho |= sto && sto->with_rho;
        maxnt = std::max(maxnt, M.nt);
    }
    if (int rc = upload_batch(plans, n, models, maps, bws, B, st)) return rc;
    const StepKernel K0 = fwd_batch_kernel_for(P0->R, fs, any_energy, any_cache ? (rho ? 2 : 1) : 0);
    if (int rc = prepare_kernel(K0)) return rc;
    const int4 *items = reinterpret_cast<const int4 *>(bws + B.items);
    const BatchModel *dmodels = reinterpret_cast<const BatchModel *>(bws + B.models);
    const BatchMaps *dmaps = reinterpret_cast<const BatchMaps *>(bws + B.maps);
    int mode = kBatchForward, t0 = 0;
    int *clock = reinterpret_cast<int *>(bws + B.clock);
    const int *no_clock = nullptr;
    P0->phase_steps[0] += maxnt;
    // a checkpoint of some model falls at step tau
    auto saves_at = [&](int tau) {
        for (int m = 0; m < n; ++m)
            if (io[m].store && tau < std::min(models[m].t_cache, models[m].nt) && tau % models[m].K == 0) return true;
        return false;
    };
    const int C = P0->graph_steps;
    int dev = -1;
    GB_CUDA(cudaGetDevice(&dev));
    const BatchLanes lanes = batch_lanes(plans, n, B.n_items);
    const std::vector<uintptr_t> key = {(uintptr_t)dev, (uintptr_t)bws, (uintptr_t)B.n_items, (uintptr_t)K0.fn,
                                        (uintptr_t)C, (uintptr_t)kBatchForward, (uintptr_t)lanes.n};
    for (int tau = 0; tau < maxnt;) {
        for (int m = 0; m < n; ++m) {
            const gb_grad_store *sto = io[m].store;
            if (sto && tau < std::min(models[m].t_cache, models[m].nt) && tau % models[m].K == 0) {
                const Layout L = layout(plans[m]);
                unsigned int *amax = reinterpret_cast<unsigned int *>(aligned_ws(io[m].workspace) + L.amax);
                if (int rc = save_checkpoint(plans[m], models[m].fld[tau & 1], sto->checkpoints, tau / models[m].K,
                                             sto->format, amax, 0, plans[m]->d.n_shots, st))
                    return rc;
            }
        }
        // chunks of C steps with no checkpoint inside: one graph replay each
        // (a checkpoint at the first step of the first chunk is saved above)
        int n_chunks = 0;
        if (C > 0)
            while (tau + (n_chunks + 1) * C <= maxnt) {
                bool clear = true;
                for (int t = tau + n_chunks * C + (n_chunks ? 0 : 1); t < tau + (n_chunks + 1) * C && clear; ++t)
                    clear = !saves_at(t);
                if (!clear) break;
                ++n_chunks;
            }
        if (n_chunks > 0) {
            if (int rc = batch_graph_chunks(P0, P0->g_batch_fwd, key, C, clock, tau, 1, n_chunks, lanes, st,
                                            [&](int j, int lane, cudaStream_t s2) {
                                                int tau_v = j;
                                                const int4 *it_l = items + lanes.off[lane];
                                                void *args[] = {(void *)&it_l, (void *)&dmodels, (void *)&dmaps,
                                                                (void *)&tau_v, (void *)&mode, (void *)&t0,
                                                                (void *)&clock};
                                                return launch_batch(P0, K0, lanes.cnt[lane], args, s2);
                                            }))
                return rc;
            tau += n_chunks * C;
            continue;
        }
        int tau_v = tau;
        void *args[] = {(void *)&items, (void *)&dmodels, (void *)&dmaps, (void *)&tau_v, (void *)&mode, (void *)&t0,
                        (void *)&no_clock};
        if (int rc = launch_batch(P0, K0, B.n_items, args, st)) return rc;
        ++tau;
    }
    for (int m = 0; m < n; ++m) {
        const gb_model_io &x = io[m];
        float *eouts[3] = {x.energy_p, x.energy_vx, x.energy_vz};
        const Layout L = layout(plans[m]);
        float *energy = reinterpret_cast<float *>(aligned_ws(x.workspace) + L.energy);
        for (int f = 0; f < 3; ++f)
            if (eouts[f]) {
                const gb_model_desc &d = plans[m]->d;
                extract_interior_kernel<<<148, 256, 0, st>>>(energy + f * plans[m]->plane, d.nz, d.nx, d.nabc,
                                                             plans[m]->pitch, eouts[f]);
                GB_CUDA(cudaGetLastError());
                ++P0->launches;
            }
    }
    P0->mark(0, false, st);
    return GB_OK;
}

int gb_batch_backward(gb_plan *const *plans, int n, const gb_model_io *io, void *batch_workspace,
                      size_t batch_workspace_bytes, void *stream)
{
    g_last_error.clear();
    if (int rc = check_batch(plans, n, io, true)) return rc;
    const BatchLayout B = batch_layout(plans, n);
    char *bws = aligned_ws(batch_workspace);
    if (!batch_workspace || batch_workspace_bytes < B.total + (size_t)(bws - reinterpret_cast<char *>(batch_workspace)))
        return fail(GB_E_WORKSPACE, "batch workspace too small");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    gb_plan *P0 = plans[0];
    const bool fs = P0->d.free_surface != 0;
    const bool rho = io[0].store->with_rho != 0;
    const int K = std::min<int>(io[0].store->checkpoint_every, 1 << 30);
    std::vector<BatchModel> models(n);
    std::vector<BatchMaps> maps(n);
    std::vector<Layout> Ls;
    int maxnt = 0;
    for (int m = 0; m < n; ++m) {
        gb_plan *P = plans[m];
        const gb_model_io &x = io[m];
        const int Km = std::min<int>(K, P->d.nt);
        // the segment buffer holds at most the uncached steps, in the store's format
        const int seg = std::max(1, std::min(Km, P->d.nt - x.store->cached_steps));
        const Layout L = layout(P, rho ? 2 : 1, seg, x.store->imaging_format);
        Ls.push_back(L);
        char *ws = aligned_ws(x.workspace);
        if (x.workspace_bytes < L.total + (size_t)(ws - reinterpret_cast<char *>(x.workspace)))
            return fail(GB_E_WORKSPACE, "workspace of model " + std::to_string(m) + " too small");
        Setup Su;
        if (int rc = common_setup(P, L, ws, x.vp, x.rho, x.damp, st, &Su)) return rc;
        const int S = P->d.n_shots;
        const size_t state_fl = (size_t)S * 3 * P->plane;
        float *fb0 = reinterpret_cast<float *>(ws + L.fields), *mu0 = reinterpret_cast<float *>(ws + L.mu);
        float *G1 = reinterpret_cast<float *>(ws + L.g1), *C1 = reinterpret_cast<float *>(ws + L.c1);
        float *G2 = rho ? reinterpret_cast<float *>(ws + L.g2) : nullptr;
        float *C2 = rho ? reinterpret_cast<float *>(ws + L.c2) : nullptr;
        int *d_aptr = reinterpret_cast<int *>(ws + L.arcv_ptr);
        int4 *d_aent = reinterpret_cast<int4 *>(ws + L.arcv_ent);
        GB_CUDA(cudaMemcpyAsync(d_aptr, P->arcv_ptr.data(), (P->n_tiles + 1) * 4, cudaMemcpyHostToDevice, st));
        if (!P->arcv_ent.empty())
            GB_CUDA(cudaMemcpyAsync(d_aent, P->arcv_ent.data(), P->arcv_ent.size() * 16, cudaMemcpyHostToDevice, st));
        GB_CUDA(cudaMemsetAsync(mu0, 0, 2 * state_fl * 4, st));
        GB_CUDA(cudaMemsetAsync(G1, 0, (size_t)P->n_groups * P->plane * 4, st));
        GB_CUDA(cudaMemsetAsync(C1, 0, (size_t)P->n_groups * P->plane * 4, st));
        if (G2) {
            GB_CUDA(cudaMemsetAsync(G2, 0, (size_t)P->n_groups * P->plane * 4, st));
            GB_CUDA(cudaMemsetAsync(C2, 0, (size_t)P->n_groups * P->plane * 4, st));
        }
        BatchModel &M = models[m];
        M = BatchModel{};
        FwdArgs &F = M.f;
        F.g = P->geom();
        F.a1 = Su.a1; F.k1 = Su.k1; F.a2 = Su.a2; F.k2 = Su.k2; F.k3 = Su.k3;
        F.tile_fast = Su.tile_fast;
        F.src_z = Su.d_src; F.src_x = Su.d_src + S;
        F.wavelet = x.wavelet;
        F.rcv_ptr = Su.d_rptr; F.rcv_ent = Su.d_rent;
        F.img_field_stride = (long long)S * P->plane;
        F.err = Su.err;
        AdjArgs &A = M.a;
        A.g = F.g;
        A.a1 = Su.a1; A.k1 = Su.k1; A.a2 = Su.a2; A.k2 = Su.k2; A.k3 = Su.k3;
        A.tile_fast = Su.tile_fast;
        A.rcv_ptr = d_aptr; A.rcv_ent = d_aent;
        A.res_p = x.res_p; A.res_vx = x.res_vx; A.res_vz = x.res_vz;
        A.img_field_stride = (long long)S * P->plane;
        A.G1 = G1; A.C1 = C1; A.G2 = G2; A.C2 = C2;
        A.err = Su.err;
        M.fld[0] = fb0;
        M.fld[1] = fb0 + state_fl;
        M.mu[0] = mu0;
        M.mu[1] = mu0 + state_fl;
        M.nt = P->d.nt;
        M.K = Km;
        M.t_cache = P->d.nt - x.store->cached_steps;
        M.cache = x.store->cached_steps > 0 ? reinterpret_cast<float *>(x.store->imaging) : nullptr;
        M.cache_fmt = x.store->imaging_format;
        M.segimg = reinterpret_cast<float *>(ws + L.img);
        M.step_img = (long long)(rho ? 3 : 1) * S * P->plane;
        if (int rc = make_state_maps(P, M.fld[0], maps[m].fld[0])) return rc;
        if (int rc = make_state_maps(P, M.fld[1], maps[m].fld[1])) return rc;
        if (int rc = make_state_maps(P, M.mu[0], maps[m].mu[0])) return rc;
        if (int rc = make_state_maps(P, M.mu[1], maps[m].mu[1])) return rc;
        if (int rc = make_map2d(&maps[m].a1, Su.a1, P->Nx, P->Nz, P->pitch, RW, box_rows_p(P->R, P->tz))) return rc;
        if (int rc = make_map2d(&maps[m].a2, Su.a2, P->Nx, P->Nz, P->pitch, RW, P->tz)) return rc;
        maxnt = std::max(maxnt, M.nt);
    }
    if (int rc = upload_batch(plans, n, models, maps, bws, B, st)) return rc;
    const StepKernel KF = fwd_batch_kernel_for(P0->R, fs, false, rho ? 2 : 1);
    int imgf = io[0].store->imaging_format;
    for (int m = 1; m < n; ++m)
        if (io[m].store->imaging_format != imgf) imgf = -1;
    const StepKernel KA = adj_batch_kernel_for(P0->R, fs, rho, imgf);
    if (int rc = prepare_kernel(KF)) return rc;
    if (int rc = prepare_kernel(KA)) return rc;
    const int4 *items = reinterpret_cast<const int4 *>(bws + B.items);
    const BatchModel *dmodels = reinterpret_cast<const BatchModel *>(bws + B.models);
    const BatchMaps *dmaps = reinterpret_cast<const BatchMaps *>(bws + B.maps);

    int *clock = reinterpret_cast<int *>(bws + B.clock);
    const int C = P0->graph_steps;
    int dev = -1;
    GB_CUDA(cudaGetDevice(&dev));
    const BatchLanes lanes = batch_lanes(plans, n, B.n_items);
    const std::vector<uintptr_t> akey = {(uintptr_t)dev, (uintptr_t)bws, (uintptr_t)B.n_items, (uintptr_t)KA.fn,
                                         (uintptr_t)C, (uintptr_t)lanes.n};
    // batch-wide segments of K steps; a model recomputes a segment only for
    // its steps below min(nt, t_cache)
    const int Kb = std::min(K, maxnt);
    const int seg_top = (maxnt - 1) / Kb;
    for (int seg = seg_top; seg >= 0; --seg) {
        const int t0 = seg * Kb, t1 = std::min(maxnt, t0 + Kb);
        int rec_end = t0;
        for (int m = 0; m < n; ++m) {
            const int lim = std::min(models[m].nt, models[m].t_cache);
            if (t0 < lim) {
                if (int rc = restore_checkpoint(plans[m], models[m].fld[0], io[m].store->checkpoints, t0 / models[m].K,
                                                io[m].store->format, 0, plans[m]->d.n_shots, st))
                    return rc;
                rec_end = std::max(rec_end, std::min(t1, lim));
            }
        }
        if (rec_end > t0) {
            P0->mark(1, true, st);
            P0->phase_steps[1] += rec_end - t0;
            int mode = kBatchRecompute, tz0 = t0;
            const int *no_clock = nullptr;
            for (int tau = t0; tau < rec_end; ++tau) {
                int tau_v = tau;
                void *args[] = {(void *)&items, (void *)&dmodels, (void *)&dmaps, (void *)&tau_v, (void *)&mode,
                                (void *)&tz0, (void *)&no_clock};
                if (int rc = launch_batch(P0, KF, B.n_items, args, st)) return rc;
            }
            P0->mark(1, false, st);
        }
        P0->mark(2, true, st);
        P0->phase_steps[2] += t1 - t0;
        int tau = t1 - 1;
        // chunks of C steps replayed from one graph (the clock counts down)
        const int n_chunks = C > 0 ? (t1 - t0) / C : 0;
        if (n_chunks > 0) {
            if (int rc = batch_graph_chunks(P0, P0->g_batch_adj, akey, C, clock, tau, -1, n_chunks, lanes, st,
                                            [&](int j, int lane, cudaStream_t s2) {
                                                int tau_v = j;
                                                const int4 *it_l = items + lanes.off[lane];
                                                void *args[] = {(void *)&it_l, (void *)&dmodels, (void *)&dmaps,
                                                                (void *)&tau_v, (void *)&clock};
                                                return launch_batch(P0, KA, lanes.cnt[lane], args, s2);
                                            }))
                return rc;
            tau -= n_chunks * C;
        }
        for (; tau >= t0; --tau) {
            int tau_v = tau;
            const int *no_clock = nullptr;
            void *args[] = {(void *)&items, (void *)&dmodels, (void *)&dmaps, (void *)&tau_v, (void *)&no_clock};
            if (int rc = launch_batch(P0, KA, B.n_items, args, st)) return rc;
        }
        P0->mark(2, false, st);
    }
    for (int m = 0; m < n; ++m) {
        const gb_model_desc &d = plans[m]->d;
        const BatchModel &M = models[m];
        grad_finish_kernel<<<4 * 148, 256, 0, st>>>(io[m].vp, io[m].rho, M.a.G1, M.a.C1, M.a.G2, M.a.C2,
                                                    plans[m]->n_groups, plans[m]->plane, d.nz, d.nx, d.nabc,
                                                    plans[m]->pitch, io[m].grad_vp, io[m].grad_rho);
        GB_CUDA(cudaGetLastError());
        ++P0->launches;
    }
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

// the array's device address per (device, context); see gb_symcache.h
gb::host::SymbolAddressCache<16> g_static_scratch_addr;

// The unique ID of the calling thread's current context (cuCtxGetCurrent and
// cuCtxGetId through the runtime's driver entry points, so that the library
// needs no link dependency on libcuda).  A thread with no current context
// gets the device's primary context made current first (cudaSetDevice); a
// context the host made current is used as it is.
using PFN_ctx_current = CUresult (*)(CUcontext *);
using PFN_ctx_id = CUresult (*)(CUcontext, unsigned long long *);
PFN_ctx_current g_ctx_current = nullptr;
PFN_ctx_id g_ctx_id = nullptr;
std::once_flag g_ctx_once;

int current_context_id(int dev, unsigned long long *id)
{
    std::call_once(g_ctx_once, [] {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qb == cudaDriverEntryPointSuccess) {
            g_ctx_current = reinterpret_cast<PFN_ctx_current>(a);
            g_ctx_id = reinterpret_cast<PFN_ctx_id>(b);
        }
    });
    if (!g_ctx_current || !g_ctx_id) return fail(GB_E_CUDA, "cuCtxGetCurrent / cuCtxGetId unavailable");
    CUcontext ctx = nullptr;
    if (g_ctx_current(&ctx) != CUDA_SUCCESS) return fail(GB_E_CUDA, "cuCtxGetCurrent failed");
    if (!ctx) {
        GB_CUDA(cudaSetDevice(dev));
        if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return fail(GB_E_CUDA, "no current CUDA context");
    }
    if (g_ctx_id(ctx, id) != CUDA_SUCCESS) return fail(GB_E_CUDA, "cuCtxGetId failed");
    return GB_OK;
}

}  // namespace

extern "C" size_t gb_static_scratch_bytes(void) { return kStaticScratchBytes; }

extern "C" int gb_forward_static_scratch(gb_plan *P, const float *vp, const float *rho, const float *damp,
                                         const float *wavelet, float *trace_p, float *trace_vx, float *trace_vz,
                                         float *energy_p, float *energy_vx, float *energy_vz,
                                         int32_t snapshot_every, float *snapshots, void *stream)
{
    g_last_error.clear();
    if (!P) return fail(GB_E_ARG, "null plan");
    // the array is 256-byte aligned, so gb_forward needs no alignment slack in it
    const size_t need = layout(P).total;
    if (need > kStaticScratchBytes)
        return fail(GB_E_WORKSPACE, "this model needs " + std::to_string(need) +
                                        " bytes of scratch; the static scratch holds " +
                                        std::to_string(kStaticScratchBytes) + " bytes (use gb_forward with a workspace)");
    int dev = -1;
    GB_CUDA(cudaGetDevice(&dev));
    unsigned long long ctx_id = 0;
    if (int rc = current_context_id(dev, &ctx_id)) return rc;
    // first call on this device and context: look the array's device address
    // up, with the device current (the host-side symbol is not a device address)
    void *scratch = nullptr;
    if (int rc = g_static_scratch_addr.get(dev, ctx_id,
                                           [](void **addr) {
                                               cudaError_t e = cudaGetSymbolAddress(addr, g_static_scratch);
                                               if (e == cudaSuccess) return 0;
                                               return fail(GB_E_CUDA,
                                                           std::string("cudaGetSymbolAddress(static scratch): ") +
                                                               cudaGetErrorString(e));
                                           },
                                           &scratch))
        return rc;
    // gb_forward clears every part of the scratch that must start at zero
    // (both wavefield time levels, the energy sums, the status word).  It
    // runs with one launch per step: instantiating a CUDA graph would make
    // the driver allocate device memory.
    const int graph_steps = P->graph_steps;
    P->graph_steps = 0;
    const int rc = gb_forward(P, vp, rho, damp, wavelet, trace_p, trace_vx, trace_vz, energy_p, energy_vx, energy_vz,
                              snapshot_every, snapshots, nullptr, scratch, kStaticScratchBytes, stream);
    P->graph_steps = graph_steps;
    return rc;
}
