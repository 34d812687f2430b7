/*
 * CPU oracle for the 2D acoustic staggered-grid propagator.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load this library, and only as
 * the checker or the timed CPU baseline.  The product path (geobrain_b200)
 * never calls it.
 *
 * What it restates (paths relative to the GeoBrain source tree):
 *   geobrain/physics/wave/kernels/acoustic_2d.py
 *     pad_model                 :18-66   edge replication            -> pad_at()
 *     coefficient preparation   :403-420 alpha1/kappa1/alpha2/kappa2/kappa3
 *     acoustic_step_forward     :123-291 one leapfrog step:
 *         p update :211-226, source :228-237, p free surface :240-241,
 *         vx update :244-253, vz update :256-265, vz free surface :268-269,
 *         receivers :272-274, energy accumulation :277-285
 *     acoustic_forward_kernel   :294-501 allocation, position shift by nabc,
 *         snapshot chunks (:422-428, :484-487)
 *   geobrain/physics/wave/kernels/elastic_2d.py:25-68 fd_coefficients(order,'s')
 *     staggered Taylor coefficients; half-width 4 gives the 8th-order set used
 *     for fd_order=8 (the reference has no 8th-order acoustic kernel; this file
 *     is the restatement the 8th-order CUDA path is checked against).
 *
 * Generalisation to stencil half-width R (R = 2 reproduces the reference
 * exactly; larger R widens only the margins the wider stencil needs):
 *     fs  = free_surface ? nabc : 1
 *     p   rows [max(fs+1, R), Nz-1-R]  cols [R,   Nx-1-R]
 *     vx  rows [fs, Nz-2]              cols [R-1, Nx-1-R]
 *     vz  rows [max(fs, R-1), Nz-1-R]  cols [1,   Nx-2]
 *     kappa2 = 0.5 (d[i,j] + d[i,j+1]) dt on cols [1, Nx-3], else 0
 *     kappa3 = 0.5 (d[i,j] + d[i+1,j]) dt on rows [fs, Nz-3], else 0
 * All fields are stored on the padded (Nz, Nx) grid; vx's last column and
 * vz's last row (absent from the reference's (Nz, Nx-1) / (Nz-1, Nx) arrays)
 * are never written or read.
 *
 * The gradient routine is the exact discrete adjoint of that step (the
 * reverse-mode graph torch.autograd builds through acoustic_step_forward and
 * pad_model), written out by hand in the unscaled form.  It keeps the state
 * before every K-th step (K = ceil(sqrt(nt))) and recomputes each segment's
 * states before running its adjoint steps, so its memory is about
 * 2 sqrt(nt) states per shot in flight.  With fewer shots than threads the
 * row loops run in parallel instead of the shots (the adjoint's scatter
 * loops in two passes over alternate blocks of rows, so that no two threads
 * add into the same cell); only the order of some additions changes.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int32_t nz, nx, nabc, nt;
    int32_t n_shots, n_rcv, half, free_surface;
    double dt, dz;
} orc_desc;

/* Staggered-grid Taylor coefficients for half-width R: solve
 *   sum_j c_j (2j+1)^(2i+1) = delta_{i0},  i,j = 0..R-1
 * (the system fd_coefficients(R, 's') builds), by Gaussian elimination in
 * double precision. */
int orc_fd_coefficients(int R, double *c)
{
    double A[8][9];
    if (R < 1 || R > 8) return -1;
    for (int i = 0; i < R; ++i) {
        for (int j = 0; j < R; ++j) A[i][j] = pow(2.0 * j + 1.0, 2.0 * i + 1.0);
        A[i][R] = (i == 0) ? 1.0 : 0.0;
    }
    for (int col = 0; col < R; ++col) {
        int piv = col;
        for (int r = col + 1; r < R; ++r)
            if (fabs(A[r][col]) > fabs(A[piv][col])) piv = r;
        if (piv != col)
            for (int k = 0; k <= R; ++k) { double t = A[col][k]; A[col][k] = A[piv][k]; A[piv][k] = t; }
        for (int r = 0; r < R; ++r) {
            if (r == col) continue;
            double f = A[r][col] / A[col][col];
            for (int k = col; k <= R; ++k) A[r][k] -= f * A[col][k];
        }
    }
    for (int i = 0; i < R; ++i) c[i] = A[i][R] / A[i][i];
    return 0;
}

int orc_max_threads(void);

/* Split the rows of each step over the threads instead of the shots: when
 * there are fewer shots than threads and the grid is large enough for the
 * per-loop thread start-up to pay (small grids keep one thread per shot). */
static int orc_split_rows(int n_shots, size_t cells)
{
    return n_shots < orc_max_threads() && cells >= ((size_t)1 << 17);
}

static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

#define REAL double
#define SFX(name) name##_f64
#include "acoustic_oracle_body.h"
#undef REAL
#undef SFX

#define REAL float
#define SFX(name) name##_f32
#include "acoustic_oracle_body.h"
#undef REAL
#undef SFX

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Thread count of the following calls (tests compare the row-split and the
 * shot-split schedules); n < 1 restores the default. */
void orc_set_threads(int n)
{
#ifdef _OPENMP
    omp_set_num_threads(n >= 1 ? n : omp_get_num_procs());
#else
    (void)n;
#endif
}
