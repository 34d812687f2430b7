/*
 * Precision-generic body of the CPU oracle (included twice by
 * acoustic_oracle.c with REAL = double and REAL = float).  TEST
 * INFRASTRUCTURE ONLY; see the header of acoustic_oracle.c for the reference
 * lines each routine restates.
 */

/* Padded coefficient arrays of acoustic_2d.py:403-420, in REAL arithmetic in
 * the reference's operation order (alpha1 = den*c*c*dt/dz, alpha2 =
 * dt/(den*dz)).  c and den are pad_model(vp/rho) (:18-66): index clamping is
 * the same edge replication. */
static void SFX(orc_coefs)(const orc_desc *d, const REAL *vp, const REAL *rho,
                           const REAL *damp, REAL *a1, REAL *a2, REAL *k1,
                           REAL *k2, REAL *k3, REAL *cpad, REAL *dpad)
{
    const int nz = d->nz, nx = d->nx, pml = d->nabc;
    const int Nz = nz + 2 * pml, Nx = nx + 2 * pml;
    const int fs = d->free_surface ? pml : 1;
    const REAL dt = (REAL)d->dt, dz = (REAL)d->dz, half = (REAL)0.5;
    for (int i = 0; i < Nz; ++i) {
        int iz = iclamp(i - pml, 0, nz - 1);
        for (int j = 0; j < Nx; ++j) {
            int ix = iclamp(j - pml, 0, nx - 1);
            REAL c = vp[(size_t)iz * nx + ix];
            REAL den = rho[(size_t)iz * nx + ix];
            size_t o = (size_t)i * Nx + j;
            cpad[o] = c;
            dpad[o] = den;
            a1[o] = den * c * c * dt / dz;
            a2[o] = dt / (den * dz);
            k1[o] = damp[o] * dt;
            k2[o] = (j >= 1 && j <= Nx - 3) ? half * (damp[o] + damp[o + 1]) * dt : (REAL)0;
            k3[o] = (i >= fs && i <= Nz - 3) ? half * (damp[o] + damp[o + Nx]) * dt : (REAL)0;
        }
    }
}

/* One leapfrog step for one shot (acoustic_2d.py:211-269), in place.  With
 * par_rows the row loops run on all threads: every update reads only other
 * fields (or the already updated pressure), so rows are independent. */
static void SFX(orc_step)(const orc_desc *d, const REAL *cf, const REAL *a1,
                          const REAL *a2, const REAL *k1, const REAL *k2,
                          const REAL *k3, REAL *p, REAL *vx, REAL *vz,
                          int spz, int spx, REAL src_amp, REAL *idiv, int par_rows)
{
    const int pml = d->nabc, R = d->half;
    const int Nz = d->nz + 2 * pml, Nx = d->nx + 2 * pml;
    const int fs = d->free_surface ? pml : 1;
    const int p_r0 = imax(fs + 1, R), p_r1 = Nz - 1 - R, p_c0 = R, p_c1 = Nx - 1 - R;
    const int vx_r0 = fs, vx_r1 = Nz - 2, vx_c0 = R - 1, vx_c1 = Nx - 1 - R;
    const int vz_r0 = imax(fs, R - 1), vz_r1 = Nz - 1 - R, vz_c0 = 1, vz_c1 = Nx - 2;

    /* pressure (:211-226) */
#pragma omp parallel for schedule(static) if(par_rows)
    for (int i = p_r0; i <= p_r1; ++i)
        for (int j = p_c0; j <= p_c1; ++j) {
            size_t o = (size_t)i * Nx + j;
            REAL D = 0;
            for (int k = 0; k < R; ++k)
                D += cf[k] * (((vx[o + k] - vx[o - 1 - k]) + vz[o + (size_t)k * Nx])
                              - vz[o - (size_t)(1 + k) * Nx]);
            if (idiv) idiv[o] = -D;
            p[o] = ((REAL)1 - k1[o]) * p[o] - a1[o] * D;
        }
    /* source (:228-237) */
    p[(size_t)spz * Nx + spx] += src_amp;
    /* free surface for p (:240-241) */
    if (d->free_surface)
        for (int j = 0; j < Nx; ++j)
            p[(size_t)(fs - 1) * Nx + j] = -p[(size_t)(fs + 1) * Nx + j];
    /* vx (:244-253) */
#pragma omp parallel for schedule(static) if(par_rows)
    for (int i = vx_r0; i <= vx_r1; ++i)
        for (int j = vx_c0; j <= vx_c1; ++j) {
            size_t o = (size_t)i * Nx + j;
            REAL D = 0;
            for (int k = 0; k < R; ++k) D += cf[k] * (p[o + 1 + k] - p[o - k]);
            vx[o] = ((REAL)1 - k2[o]) * vx[o] - a2[o] * D;
        }
    /* vz (:256-265) */
#pragma omp parallel for schedule(static) if(par_rows)
    for (int i = vz_r0; i <= vz_r1; ++i)
        for (int j = vz_c0; j <= vz_c1; ++j) {
            size_t o = (size_t)i * Nx + j;
            REAL D = 0;
            for (int k = 0; k < R; ++k)
                D += cf[k] * (p[o + (size_t)(1 + k) * Nx] - p[o - (size_t)k * Nx]);
            vz[o] = ((REAL)1 - k3[o]) * vz[o] - a2[o] * D;
        }
    /* free surface for vz (:268-269) */
    if (d->free_surface)
        for (int j = 0; j < Nx; ++j)
            vz[(size_t)(fs - 1) * Nx + j] = vz[(size_t)fs * Nx + j];
}

static int SFX(orc_check_positions)(const orc_desc *d, const int64_t *sx, const int64_t *sz,
                                    const int64_t *rx, const int64_t *rz)
{
    for (int s = 0; s < d->n_shots; ++s)
        if (sx[s] < -d->nabc || sx[s] >= d->nx + d->nabc || sz[s] < -d->nabc || sz[s] >= d->nz + d->nabc)
            return -2;
    for (int r = 0; r < d->n_rcv; ++r)
        if (rx[r] < -d->nabc || rx[r] >= d->nx + d->nabc - 1 || rz[r] < -d->nabc || rz[r] >= d->nz + d->nabc - 1)
            return -2;
    return 0;
}

/* Forward modelling (acoustic_forward_kernel, :294-501).  Positions are the
 * unpadded grid indices the reference takes; traces are (n_shots, nt, n_rcv),
 * energies (nz, nx); snapshots (ceil(nt/snapshot_every), nz, nx) of shot 0
 * taken at the end of each snapshot chunk (:422-428, :484-487). */
int SFX(orc_forward)(const orc_desc *d, const REAL *vp, const REAL *rho, const REAL *damp,
                     const int64_t *sx, const int64_t *sz, const REAL *wav,
                     const int64_t *rx, const int64_t *rz,
                     REAL *tr_p, REAL *tr_vx, REAL *tr_vz,
                     REAL *en_p, REAL *en_vx, REAL *en_vz,
                     int snapshot_every, REAL *snaps)
{
    const int nz = d->nz, nx = d->nx, pml = d->nabc, nt = d->nt, S = d->n_shots, NR = d->n_rcv;
    const int Nz = nz + 2 * pml, Nx = nx + 2 * pml;
    const size_t NN = (size_t)Nz * Nx;
    double cfd[8];
    REAL cf[8];
    if (d->half < 1 || d->half > 8 || pml < d->half) return -1;
    if (SFX(orc_check_positions)(d, sx, sz, rx, rz)) return -2;
    orc_fd_coefficients(d->half, cfd);
    if (d->half == 2) { cfd[0] = 9.0 / 8.0; cfd[1] = -1.0 / 24.0; }  /* :403-404 */
    for (int k = 0; k < d->half; ++k) cf[k] = (REAL)cfd[k];

    REAL *buf = (REAL *)calloc(NN * (7 + 3 * (size_t)S), sizeof(REAL));
    if (!buf) return -3;
    REAL *a1 = buf, *a2 = a1 + NN, *k1 = a2 + NN, *k2 = k1 + NN, *k3 = k2 + NN;
    REAL *cpad = k3 + NN, *dpad = cpad + NN, *F = dpad + NN;
    SFX(orc_coefs)(d, vp, rho, damp, a1, a2, k1, k2, k3, cpad, dpad);
    memset(en_p, 0, sizeof(REAL) * nz * nx);
    memset(en_vx, 0, sizeof(REAL) * nz * nx);
    memset(en_vz, 0, sizeof(REAL) * nz * nx);
    const REAL dt = (REAL)d->dt;
    const int par_rows = orc_split_rows(S, NN);
    int snap_i = 0;
    for (int it = 0; it < nt; ++it) {
#pragma omp parallel for schedule(static) if(!par_rows)
        for (int s = 0; s < S; ++s) {
            REAL *p = F + (size_t)s * 3 * NN, *vx = p + NN, *vz = vx + NN;
            SFX(orc_step)(d, cf, a1, a2, k1, k2, k3, p, vx, vz,
                          (int)sz[s] + pml, (int)sx[s] + pml, dt * wav[(size_t)s * nt + it], NULL, par_rows);
            for (int r = 0; r < NR; ++r) {
                size_t o = (size_t)(rz[r] + pml) * Nx + (rx[r] + pml);
                size_t t = ((size_t)s * nt + it) * NR + r;
                tr_p[t] = p[o];
                tr_vx[t] = vx[o];
                tr_vz[t] = vz[o];
            }
        }
        /* energies: sum over shots of the squared interior fields (:277-285) */
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz)
            for (int ix = 0; ix < nx; ++ix) {
                size_t o = (size_t)(iz + pml) * Nx + (ix + pml);
                REAL ep = 0, ex = 0, ez = 0;
                for (int s = 0; s < S; ++s) {
                    const REAL *p = F + (size_t)s * 3 * NN;
                    ep += p[o] * p[o];
                    ex += p[NN + o] * p[NN + o];
                    ez += p[2 * NN + o] * p[2 * NN + o];
                }
                en_p[(size_t)iz * nx + ix] += ep;
                en_vx[(size_t)iz * nx + ix] += ex;
                en_vz[(size_t)iz * nx + ix] += ez;
            }
        if (snapshot_every > 0 && snaps && ((it + 1) % snapshot_every == 0 || it == nt - 1)) {
            for (int iz = 0; iz < nz; ++iz)
                for (int ix = 0; ix < nx; ++ix)
                    snaps[((size_t)snap_i * nz + iz) * nx + ix] = F[(size_t)(iz + pml) * Nx + ix + pml];
            ++snap_i;
        }
    }
    free(buf);
    return 0;
}

/* Gradient of L with respect to vp and rho (and the wavelet) given the
 * adjoint sources dL/d(trace) res_* (n_shots, nt, n_rcv): the discrete
 * adjoint of every forward stage above, run backwards in time over the
 * forward states (recomputed a segment at a time from stored ones), then the adjoint of pad_model (edge cells collect the
 * gradient of the padding they were replicated into).  g_vp, g_rho are
 * (nz, nx); g_wav (n_shots, nt) may be NULL. */
int SFX(orc_gradient)(const orc_desc *d, const REAL *vp, const REAL *rho, const REAL *damp,
                      const int64_t *sx, const int64_t *sz, const REAL *wav,
                      const int64_t *rx, const int64_t *rz,
                      const REAL *res_p, const REAL *res_vx, const REAL *res_vz,
                      REAL *g_vp, REAL *g_rho, REAL *g_wav)
{
    const int nz = d->nz, nx = d->nx, pml = d->nabc, nt = d->nt, S = d->n_shots, NR = d->n_rcv;
    const int R = d->half;
    const int Nz = nz + 2 * pml, Nx = nx + 2 * pml;
    const size_t NN = (size_t)Nz * Nx;
    const int fs = d->free_surface ? pml : 1;
    const int p_r0 = imax(fs + 1, R), p_r1 = Nz - 1 - R, p_c0 = R, p_c1 = Nx - 1 - R;
    const int vx_r0 = fs, vx_r1 = Nz - 2, vx_c0 = R - 1, vx_c1 = Nx - 1 - R;
    const int vz_r0 = imax(fs, R - 1), vz_r1 = Nz - 1 - R, vz_c0 = 1, vz_c1 = Nx - 2;
    double cfd[8];
    REAL cf[8];
    if (R < 1 || R > 8 || pml < R) return -1;
    if (SFX(orc_check_positions)(d, sx, sz, rx, rz)) return -2;
    orc_fd_coefficients(R, cfd);
    if (R == 2) { cfd[0] = 9.0 / 8.0; cfd[1] = -1.0 / 24.0; }
    for (int k = 0; k < R; ++k) cf[k] = (REAL)cfd[k];
    const REAL dt = (REAL)d->dt, dz = (REAL)d->dz;

    REAL *coef = (REAL *)calloc(NN * 7, sizeof(REAL));
    REAL *work = (REAL *)calloc(NN * 7 * (size_t)S, sizeof(REAL));
    if (!coef || !work) { free(coef); free(work); return -3; }
    REAL *a1 = coef, *a2 = a1 + NN, *k1 = a2 + NN, *k2 = k1 + NN, *k3 = k2 + NN;
    REAL *cpad = k3 + NN, *dpad = cpad + NN;
    SFX(orc_coefs)(d, vp, rho, damp, a1, a2, k1, k2, k3, cpad, dpad);
    /* segment length of the stored states, and how the threads split */
    int Kc = 1;
    while ((long long)Kc * Kc < nt) ++Kc;
    const int n_ck = (nt + Kc - 1) / Kc;
    const int par_rows = orc_split_rows(S, NN);
    /* blocks of rows for the scatter loops: a row's updates reach at most R
     * rows either side, so blocks of at least 2R rows, two apart, never touch
     * the same cell */
    const int B = 16 > 2 * R ? 16 : 2 * R;

    int err = 0;
#pragma omp parallel for schedule(static) if(!par_rows)
    for (int s = 0; s < S; ++s) {
        REAL *p = work + (size_t)s * 7 * NN, *vx = p + NN, *vz = vx + NN;
        REAL *lp = vz + NN, *lvx = lp + NN, *lvz = lvx + NN, *idv = lvz + NN;
        REAL *ga1 = (REAL *)calloc(NN * 2, sizeof(REAL));
        REAL *ck = (REAL *)malloc(sizeof(REAL) * 3 * NN * (size_t)n_ck);
        REAL *seg = (REAL *)malloc(sizeof(REAL) * 3 * NN * (size_t)Kc);
        REAL *tvx = (REAL *)malloc(sizeof(REAL) * 2 * NN);
        if (!ga1 || !ck || !seg || !tvx) {
            err = -3;
            free(ga1); free(ck); free(seg); free(tvx);
            continue;
        }
        REAL *ga2 = ga1 + NN;
        const int spz = (int)sz[s] + pml, spx = (int)sx[s] + pml;
        /* forward, keeping the state before every Kc-th step */
        for (int it = 0; it < nt; ++it) {
            if (it % Kc == 0) memcpy(ck + (size_t)(it / Kc) * 3 * NN, p, sizeof(REAL) * 3 * NN);
            SFX(orc_step)(d, cf, a1, a2, k1, k2, k3, p, vx, vz, spz, spx,
                          dt * wav[(size_t)s * nt + it], NULL, par_rows);
        }
        memset(lp, 0, sizeof(REAL) * 3 * NN);
        for (int c = n_ck - 1; c >= 0; --c) {
            const int t0 = c * Kc, t1 = t0 + Kc < nt ? t0 + Kc : nt;
            /* recompute the segment's states from its stored state */
            memcpy(p, ck + (size_t)c * 3 * NN, sizeof(REAL) * 3 * NN);
            for (int it = t0; it < t1; ++it) {
                memcpy(seg + (size_t)(it - t0) * 3 * NN, p, sizeof(REAL) * 3 * NN);
                SFX(orc_step)(d, cf, a1, a2, k1, k2, k3, p, vx, vz, spz, spx,
                              dt * wav[(size_t)s * nt + it], NULL, par_rows);
            }
            for (int it = t1 - 1; it >= t0; --it) {
                /* rebuild the state before step it, and p3 (p after update,
                 * source and free surface) and -Dv(v^it) from it */
                memcpy(p, seg + (size_t)(it - t0) * 3 * NN, sizeof(REAL) * 3 * NN);
                memcpy(tvx, vx, sizeof(REAL) * 2 * NN);
                SFX(orc_step)(d, cf, a1, a2, k1, k2, k3, p, tvx, tvx + NN, spz, spx,
                              dt * wav[(size_t)s * nt + it], idv, par_rows);
                /* p now holds p3; vx, vz hold the pre-step velocities */
                /* receivers (:272-274): gather -> scatter-add of the residuals */
                for (int r = 0; r < NR; ++r) {
                    size_t o = (size_t)(rz[r] + pml) * Nx + (rx[r] + pml);
                    size_t t = ((size_t)s * nt + it) * NR + r;
                    lp[o] += res_p[t];
                    lvx[o] += res_vx[t];
                    lvz[o] += res_vz[t];
                }
                /* vz free surface (:268-269) */
                if (d->free_surface)
                    for (int j = 0; j < Nx; ++j) {
                        lvz[(size_t)fs * Nx + j] += lvz[(size_t)(fs - 1) * Nx + j];
                        lvz[(size_t)(fs - 1) * Nx + j] = 0;
                    }
                /* vz update (:256-265); it adds into lp up to R rows away */
                for (int color = 0; color < 2; ++color) {
                    const int nblk = (vz_r1 - vz_r0 + B) / B;
#pragma omp parallel for schedule(static) if(par_rows)
                    for (int b = color; b < nblk; b += 2) {
                        const int i0 = vz_r0 + b * B, i1 = i0 + B - 1 < vz_r1 ? i0 + B - 1 : vz_r1;
                        for (int i = i0; i <= i1; ++i)
                            for (int j = vz_c0; j <= vz_c1; ++j) {
                                size_t o = (size_t)i * Nx + j;
                                REAL q = lvz[o], D = 0;
                                for (int k = 0; k < R; ++k) {
                                    D += cf[k] * (p[o + (size_t)(1 + k) * Nx] - p[o - (size_t)k * Nx]);
                                    lp[o + (size_t)(1 + k) * Nx] -= a2[o] * cf[k] * q;
                                    lp[o - (size_t)k * Nx] += a2[o] * cf[k] * q;
                                }
                                ga2[o] -= q * D;
                                lvz[o] = ((REAL)1 - k3[o]) * q;
                            }
                    }
                }
                /* vx update (:244-253); its additions stay in the row */
#pragma omp parallel for schedule(static) if(par_rows)
                for (int i = vx_r0; i <= vx_r1; ++i)
                    for (int j = vx_c0; j <= vx_c1; ++j) {
                        size_t o = (size_t)i * Nx + j;
                        REAL q = lvx[o], D = 0;
                        for (int k = 0; k < R; ++k) {
                            D += cf[k] * (p[o + 1 + k] - p[o - k]);
                            lp[o + 1 + k] -= a2[o] * cf[k] * q;
                            lp[o - k] += a2[o] * cf[k] * q;
                        }
                        ga2[o] -= q * D;
                        lvx[o] = ((REAL)1 - k2[o]) * q;
                    }
                /* p free surface (:240-241) */
                if (d->free_surface)
                    for (int j = 0; j < Nx; ++j) {
                        lp[(size_t)(fs + 1) * Nx + j] -= lp[(size_t)(fs - 1) * Nx + j];
                        lp[(size_t)(fs - 1) * Nx + j] = 0;
                    }
                /* source (:228-237) */
                if (g_wav) g_wav[(size_t)s * nt + it] = dt * lp[(size_t)spz * Nx + spx];
                /* p update (:211-226); it adds into lvz up to R rows away */
                for (int color = 0; color < 2; ++color) {
                    const int nblk = (p_r1 - p_r0 + B) / B;
#pragma omp parallel for schedule(static) if(par_rows)
                    for (int b = color; b < nblk; b += 2) {
                        const int i0 = p_r0 + b * B, i1 = i0 + B - 1 < p_r1 ? i0 + B - 1 : p_r1;
                        for (int i = i0; i <= i1; ++i)
                            for (int j = p_c0; j <= p_c1; ++j) {
                                size_t o = (size_t)i * Nx + j;
                                REAL q = lp[o];
                                REAL w = a1[o] * q;
                                ga1[o] += q * idv[o];
                                for (int k = 0; k < R; ++k) {
                                    lvx[o + k] -= cf[k] * w;
                                    lvx[o - 1 - k] += cf[k] * w;
                                    lvz[o + (size_t)k * Nx] -= cf[k] * w;
                                    lvz[o - (size_t)(1 + k) * Nx] += cf[k] * w;
                                }
                                lp[o] = ((REAL)1 - k1[o]) * q;
                            }
                    }
                }
            }
        }
        /* alpha1 = den c^2 dt/dz, alpha2 = dt/(den dz) -> c, den */
        for (size_t o = 0; o < NN; ++o) {
            REAL c = cpad[o], den = dpad[o];
            REAL gc = ga1[o] * ((REAL)2 * den * c * dt / dz);
            REAL gd = ga1[o] * (c * c * dt / dz) - ga2[o] * (dt / (den * den * dz));
            ga1[o] = gc;
            ga2[o] = gd;
        }
        /* park the per-shot padded gradients in the (now unused) idv/lp slots */
        memcpy(lp, ga1, sizeof(REAL) * NN);
        memcpy(lvx, ga2, sizeof(REAL) * NN);
        free(ga1); free(ck); free(seg); free(tvx);
    }
    if (err) { free(coef); free(work); return err; }
    /* sum over shots, then fold the padding into the edge cells (pad_model
     * adjoint) */
    memset(g_vp, 0, sizeof(REAL) * nz * nx);
    memset(g_rho, 0, sizeof(REAL) * nz * nx);
    for (int s = 0; s < S; ++s) {
        const REAL *gc = work + (size_t)s * 7 * NN + 3 * NN, *gd = gc + NN;
        for (int i = 0; i < Nz; ++i) {
            int iz = iclamp(i - pml, 0, nz - 1);
            for (int j = 0; j < Nx; ++j) {
                int ix = iclamp(j - pml, 0, nx - 1);
                g_vp[(size_t)iz * nx + ix] += gc[(size_t)i * Nx + j];
                g_rho[(size_t)iz * nx + ix] += gd[(size_t)i * Nx + j];
            }
        }
    }
    free(coef); free(work);
    return 0;
}
