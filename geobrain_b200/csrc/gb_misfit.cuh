// Trace-normalised L2 misfit of GeoBrain's FWI example and its adjoint
// source, on the device (examples/09_acoustic_fwi.py:290-319):
//   m_d = max(max_t |d_t|, 1e-30), m_o likewise
//   r_t = o_t / m_o - d_t / m_d,   L_j = sqrt(sum_t r_t^2)
//   loss = sum of L_j over traces not silent in both d and o
// and dloss/dd_t = g_t / m_d - [t == t*] sign(d_t*) (sum_u g_u d_u) / m_d^2
// with g_t = -r_t / L_j and t* the first index of the largest |d_t| (the
// max's own gradient, absent when max |d| < 1e-30).  Silent traces and
// traces with L_j = 0 get a zero adjoint source.
//
// One thread per trace (shot, receiver); for each time sample the 32 lanes
// of a warp read 32 adjacent receivers (coalesced).  Three passes over the
// trace: maxima and silence, residual sums, adjoint source.  Sums run in
// fp64; the normalisation divides in fp32 as the example does.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gb {

constexpr float kMisfitClamp = 1e-30f;

__global__ void __launch_bounds__(128)
trace_misfit_kernel(const float *__restrict__ pred, const float *__restrict__ obs, int nt, int n_rcv,
                    float *__restrict__ adj, float *__restrict__ per_trace)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (r >= n_rcv) return;
    const long long base = (long long)s * nt * n_rcv + r;
    const float *d = pred + base;
    const float *o = obs + base;

    float max_d = 0.f, max_o = 0.f;
    int t_star = 0;
    bool live_d = false, live_o = false;
    for (int t = 0; t < nt; ++t) {
        const float dv = d[(long long)t * n_rcv], ov = o[(long long)t * n_rcv];
        const float ad = fabsf(dv);
        if (ad > max_d) {            // strict: the first index of the maximum keeps it
            max_d = ad;
            t_star = t;
        }
        max_o = fmaxf(max_o, fabsf(ov));
        live_d |= dv != 0.f;
        live_o |= ov != 0.f;
    }
    const bool active = live_d || live_o;
    const float m_d = fmaxf(max_d, kMisfitClamp), m_o = fmaxf(max_o, kMisfitClamp);

    double r2 = 0.0, rd = 0.0;
    for (int t = 0; t < nt; ++t) {
        const float dv = d[(long long)t * n_rcv];
        const float rv = __fsub_rn(__fdiv_rn(o[(long long)t * n_rcv], m_o), __fdiv_rn(dv, m_d));
        r2 = fma((double)rv, (double)rv, r2);
        rd = fma((double)rv, (double)dv, rd);
    }
    const double L = sqrt(r2);
    per_trace[(long long)s * n_rcv + r] = active ? (float)L : 0.f;
    if (!adj) return;
    float *a = adj + base;
    if (!active || L == 0.0) {
        for (int t = 0; t < nt; ++t) a[(long long)t * n_rcv] = 0.f;
        return;
    }
    // sum_u g_u d_u = -(sum_u r_u d_u) / L; the max's term lands on t*
    const double inv_l = 1.0 / L;
    const double corr = max_d >= kMisfitClamp
                            ? (d[(long long)t_star * n_rcv] > 0.f ? 1.0 : -1.0) * (-rd * inv_l) / ((double)m_d * m_d)
                            : 0.0;
    for (int t = 0; t < nt; ++t) {
        const float dv = d[(long long)t * n_rcv];
        const float rv = __fsub_rn(__fdiv_rn(o[(long long)t * n_rcv], m_o), __fdiv_rn(dv, m_d));
        double g = -(double)rv * inv_l / (double)m_d;
        if (t == t_star) g -= corr;
        a[(long long)t * n_rcv] = (float)g;
    }
}

// loss = sum of the per-trace values, in a fixed order (deterministic).
__global__ void __launch_bounds__(1024) trace_misfit_sum_kernel(const float *__restrict__ per_trace, long long n,
                                                               float *__restrict__ loss)
{
    __shared__ double part[1024];
    double acc = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) acc += (double)per_trace[i];
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = (float)part[0];
}

}  // namespace gb
