"""CPU oracle of the 3-D acoustic forward kernel, in NumPy.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA 3-D
path; the product package never imports it.

Restates geobrain/physics/wave/kernels/acoustic_3d.py (the step :20-300,
the driver :303-476, pad_model_3d at kernels/acoustic_2d.py:70-120) with
whole-array NumPy operations, in float64 or float32, for small grids.
Positions are the unpadded indices the reference takes (it adds nabc).
"""
from __future__ import annotations

import numpy as np

C1, C2 = 9.0 / 8.0, -1.0 / 24.0


def pad3(v: np.ndarray, pml: int) -> np.ndarray:
    """Edge replication on all six faces (pad_model_3d)."""
    return np.pad(v, pml, mode="edge")


def forward(*, nz, ny, nx, dz, nt, dt, nabc, free_surface, src_x, src_y, src_z, src_v, rcv_x, rcv_y, rcv_z,
            damp, vp, rho, dtype=np.float64):
    t = dtype
    c = pad3(np.asarray(vp, t), nabc)
    den = pad3(np.asarray(rho, t), nabc)
    damp = np.asarray(damp, t)
    dt, dz = t(dt), t(dz)
    fs = nabc if free_surface else 1
    Nz, Ny, Nx = nz + 2 * nabc, ny + 2 * nabc, nx + 2 * nabc
    c1, c2 = t(C1), t(C2)
    # coefficients (acoustic_3d.py:410-441)
    a1 = den * c * c * dt / dz
    k1 = damp * dt
    a2 = dt / (den * dz)
    k2 = np.zeros_like(damp)
    k2[:, :, 1:Nx - 2] = t(0.5) * (damp[:, :, 1:Nx - 2] + damp[:, :, 2:Nx - 1]) * dt
    k3 = np.zeros_like(damp)
    k3[:, 1:Ny - 2, :] = t(0.5) * (damp[:, 1:Ny - 2, :] + damp[:, 2:Ny - 1, :]) * dt
    k4 = np.zeros_like(damp)
    k4[fs:Nz - 2] = t(0.5) * (damp[fs:Nz - 2] + damp[fs + 1:Nz - 1]) * dt

    S = len(src_x)
    sx, sy, sz = (np.asarray(a, np.int64) + nabc for a in (src_x, src_y, src_z))
    rx, ry, rz = (np.asarray(a, np.int64) + nabc for a in (rcv_x, rcv_y, rcv_z))
    w = np.asarray(src_v, t)
    p = np.zeros((S, Nz, Ny, Nx), t)
    vx = np.zeros((S, Nz, Ny, Nx - 1), t)
    vy = np.zeros((S, Nz, Ny - 1, Nx), t)
    vz = np.zeros((S, Nz - 1, Ny, Nx), t)
    tr = {k: np.zeros((S, nt, len(rx)), t) for k in ("p", "vx", "vy", "vz")}
    en = {k: np.zeros((nz, ny, nx), t) for k in ("p", "vx", "vy", "vz")}
    z0, z1, y0, y1, x0, x1 = fs + 1, Nz - 2, 2, Ny - 2, 2, Nx - 2
    for it in range(nt):
        # pressure (:117-150)
        dvx = (c1 * (vx[:, z0:z1, y0:y1, x0:x1] - vx[:, z0:z1, y0:y1, x0 - 1:x1 - 1]) +
               c2 * (vx[:, z0:z1, y0:y1, x0 + 1:x1 + 1] - vx[:, z0:z1, y0:y1, x0 - 2:x1 - 2]))
        dvy = (c1 * (vy[:, z0:z1, y0:y1, x0:x1] - vy[:, z0:z1, y0 - 1:y1 - 1, x0:x1]) +
               c2 * (vy[:, z0:z1, y0 + 1:y1 + 1, x0:x1] - vy[:, z0:z1, y0 - 2:y1 - 2, x0:x1]))
        dvz = (c1 * (vz[:, z0:z1, y0:y1, x0:x1] - vz[:, z0 - 1:z1 - 1, y0:y1, x0:x1]) +
               c2 * (vz[:, z0 + 1:z1 + 1, y0:y1, x0:x1] - vz[:, z0 - 2:z1 - 2, y0:y1, x0:x1]))
        p[:, z0:z1, y0:y1, x0:x1] = ((t(1) - k1[z0:z1, y0:y1, x0:x1]) * p[:, z0:z1, y0:y1, x0:x1] -
                                     a1[z0:z1, y0:y1, x0:x1] * (dvx + dvy + dvz))
        # source (:153-163) and free surface (:166-167)
        p[np.arange(S), sz, sy, sx] += dt * w[:, it]
        if free_surface:
            p[:, fs - 1] = -p[:, fs + 1]
        # velocities (:170-233)
        zs, ze = fs, Nz - 1
        vx[:, zs:ze, 1:Ny - 1, 1:Nx - 2] = (
            (t(1) - k2[zs:ze, 1:Ny - 1, 1:Nx - 2]) * vx[:, zs:ze, 1:Ny - 1, 1:Nx - 2] -
            a2[zs:ze, 1:Ny - 1, 1:Nx - 2] * (c1 * (p[:, zs:ze, 1:Ny - 1, 2:Nx - 1] - p[:, zs:ze, 1:Ny - 1, 1:Nx - 2]) +
                                             c2 * (p[:, zs:ze, 1:Ny - 1, 3:Nx] - p[:, zs:ze, 1:Ny - 1, 0:Nx - 3])))
        vy[:, zs:ze, 1:Ny - 2, 1:Nx - 1] = (
            (t(1) - k3[zs:ze, 1:Ny - 2, 1:Nx - 1]) * vy[:, zs:ze, 1:Ny - 2, 1:Nx - 1] -
            a2[zs:ze, 1:Ny - 2, 1:Nx - 1] * (c1 * (p[:, zs:ze, 2:Ny - 1, 1:Nx - 1] - p[:, zs:ze, 1:Ny - 2, 1:Nx - 1]) +
                                             c2 * (p[:, zs:ze, 3:Ny, 1:Nx - 1] - p[:, zs:ze, 0:Ny - 3, 1:Nx - 1])))
        ze = Nz - 2
        vz[:, zs:ze, 1:Ny - 1, 1:Nx - 1] = (
            (t(1) - k4[zs:ze, 1:Ny - 1, 1:Nx - 1]) * vz[:, zs:ze, 1:Ny - 1, 1:Nx - 1] -
            a2[zs:ze, 1:Ny - 1, 1:Nx - 1] * (c1 * (p[:, zs + 1:ze + 1, 1:Ny - 1, 1:Nx - 1] - p[:, zs:ze, 1:Ny - 1, 1:Nx - 1]) +
                                             c2 * (p[:, zs + 2:ze + 2, 1:Ny - 1, 1:Nx - 1] - p[:, zs - 1:ze - 1, 1:Ny - 1, 1:Nx - 1])))
        if free_surface:
            vz[:, fs - 1] = vz[:, fs]
        # receivers (:240-243) and energy (:246-258)
        for k, f in (("p", p), ("vx", vx), ("vy", vy), ("vz", vz)):
            tr[k][:, it, :] = f[:, rz, ry, rx]
            en[k] += (f * f).sum(axis=0)[nabc:nabc + nz, nabc:nabc + ny, nabc:nabc + nx]
    out = {k: v for k, v in tr.items()}
    out.update({f"forward_wavefield_{k}": v for k, v in en.items()})
    return out


def gradient(*, nz, ny, nx, dz, nt, dt, nabc, free_surface, src_x, src_y, src_z, src_v, rcv_x, rcv_y, rcv_z,
             damp, vp, rho, res_p=None, res_vx=None, res_vy=None, res_vz=None, with_wavelet=False):
    """dL/dvp and dL/drho (nz, ny, nx), float64 (and, with_wavelet,
    dL/dsrc_v (shots, nt): dt times the adjoint of p just after the source
    was added, acoustic_3d.py:153-163), for the adjoint sources
    res_* = dL/d(trace_*) (shots, nt, receivers): the exact discrete adjoint
    of forward() run backwards in time over the stored states (the
    transposed p / v updates, the free-surface folds, the receiver
    injections), then the chain rule through a1 = rho c^2 dt / dz,
    a2 = dt / (rho dz) and the fold of pad_model_3d."""
    t = np.float64
    c = pad3(np.asarray(vp, t), nabc)
    den = pad3(np.asarray(rho, t), nabc)
    damp = np.asarray(damp, t)
    fs = nabc if free_surface else 1
    Nz, Ny, Nx = nz + 2 * nabc, ny + 2 * nabc, nx + 2 * nabc
    c1, c2 = C1, C2
    a1 = den * c * c * dt / dz
    k1 = damp * dt
    a2 = dt / (den * dz)
    k2 = np.zeros_like(damp)
    k2[:, :, 1:Nx - 2] = 0.5 * (damp[:, :, 1:Nx - 2] + damp[:, :, 2:Nx - 1]) * dt
    k3 = np.zeros_like(damp)
    k3[:, 1:Ny - 2, :] = 0.5 * (damp[:, 1:Ny - 2, :] + damp[:, 2:Ny - 1, :]) * dt
    k4 = np.zeros_like(damp)
    k4[fs:Nz - 2] = 0.5 * (damp[fs:Nz - 2] + damp[fs + 1:Nz - 1]) * dt
    S = len(src_x)
    sx, sy, sz = (np.asarray(a, np.int64) + nabc for a in (src_x, src_y, src_z))
    rx, ry, rz = (np.asarray(a, np.int64) + nabc for a in (rcv_x, rcv_y, rcv_z))
    w = np.asarray(src_v, t)
    p = np.zeros((S, Nz, Ny, Nx), t)
    vx = np.zeros((S, Nz, Ny, Nx - 1), t)
    vy = np.zeros((S, Nz, Ny - 1, Nx), t)
    vz = np.zeros((S, Nz - 1, Ny, Nx), t)
    z0, z1, y0, y1, x0, x1 = fs + 1, Nz - 2, 2, Ny - 2, 2, Nx - 2
    hist_v, hist_p = [], []          # v^n (before step n) and p^{n+1} (after step n's p update and mirror)
    for it in range(nt):
        hist_v.append((vx.copy(), vy.copy(), vz.copy()))
        dvx = (c1 * (vx[:, z0:z1, y0:y1, x0:x1] - vx[:, z0:z1, y0:y1, x0 - 1:x1 - 1]) +
               c2 * (vx[:, z0:z1, y0:y1, x0 + 1:x1 + 1] - vx[:, z0:z1, y0:y1, x0 - 2:x1 - 2]))
        dvy = (c1 * (vy[:, z0:z1, y0:y1, x0:x1] - vy[:, z0:z1, y0 - 1:y1 - 1, x0:x1]) +
               c2 * (vy[:, z0:z1, y0 + 1:y1 + 1, x0:x1] - vy[:, z0:z1, y0 - 2:y1 - 2, x0:x1]))
        dvz = (c1 * (vz[:, z0:z1, y0:y1, x0:x1] - vz[:, z0 - 1:z1 - 1, y0:y1, x0:x1]) +
               c2 * (vz[:, z0 + 1:z1 + 1, y0:y1, x0:x1] - vz[:, z0 - 2:z1 - 2, y0:y1, x0:x1]))
        p[:, z0:z1, y0:y1, x0:x1] = ((1 - k1[z0:z1, y0:y1, x0:x1]) * p[:, z0:z1, y0:y1, x0:x1] -
                                     a1[z0:z1, y0:y1, x0:x1] * (dvx + dvy + dvz))
        p[np.arange(S), sz, sy, sx] += dt * w[:, it]
        if free_surface:
            p[:, fs - 1] = -p[:, fs + 1]
        hist_p.append(p.copy())
        zs, ze = fs, Nz - 1
        vx[:, zs:ze, 1:Ny - 1, 1:Nx - 2] = (
            (1 - k2[zs:ze, 1:Ny - 1, 1:Nx - 2]) * vx[:, zs:ze, 1:Ny - 1, 1:Nx - 2] -
            a2[zs:ze, 1:Ny - 1, 1:Nx - 2] * (c1 * (p[:, zs:ze, 1:Ny - 1, 2:Nx - 1] - p[:, zs:ze, 1:Ny - 1, 1:Nx - 2]) +
                                             c2 * (p[:, zs:ze, 1:Ny - 1, 3:Nx] - p[:, zs:ze, 1:Ny - 1, 0:Nx - 3])))
        vy[:, zs:ze, 1:Ny - 2, 1:Nx - 1] = (
            (1 - k3[zs:ze, 1:Ny - 2, 1:Nx - 1]) * vy[:, zs:ze, 1:Ny - 2, 1:Nx - 1] -
            a2[zs:ze, 1:Ny - 2, 1:Nx - 1] * (c1 * (p[:, zs:ze, 2:Ny - 1, 1:Nx - 1] - p[:, zs:ze, 1:Ny - 2, 1:Nx - 1]) +
                                             c2 * (p[:, zs:ze, 3:Ny, 1:Nx - 1] - p[:, zs:ze, 0:Ny - 3, 1:Nx - 1])))
        vz[:, fs:Nz - 2, 1:Ny - 1, 1:Nx - 1] = (
            (1 - k4[fs:Nz - 2, 1:Ny - 1, 1:Nx - 1]) * vz[:, fs:Nz - 2, 1:Ny - 1, 1:Nx - 1] -
            a2[fs:Nz - 2, 1:Ny - 1, 1:Nx - 1] * (
                c1 * (p[:, fs + 1:Nz - 1, 1:Ny - 1, 1:Nx - 1] - p[:, fs:Nz - 2, 1:Ny - 1, 1:Nx - 1]) +
                c2 * (p[:, fs + 2:Nz, 1:Ny - 1, 1:Nx - 1] - p[:, fs - 1:Nz - 3, 1:Ny - 1, 1:Nx - 1])))
        if free_surface:
            vz[:, fs - 1] = vz[:, fs]

    zero = np.zeros((S, nt, len(rx)))
    res = [np.asarray(r, t) if r is not None else zero for r in (res_p, res_vx, res_vy, res_vz)]
    lp, lx, ly, lz = np.zeros_like(p), np.zeros_like(vx), np.zeros_like(vy), np.zeros_like(vz)
    gw = np.zeros((S, nt))             # dL/dsrc_v
    g1 = np.zeros((Nz, Ny, Nx))       # dL/da1
    g2 = np.zeros((Nz, Ny, Nx))       # dL/da2
    si = np.arange(S)[:, None]
    for it in range(nt - 1, -1, -1):
        # adjoint of the recording of step it
        for lam, r in ((lp, res[0]), (lx, res[1]), (ly, res[2]), (lz, res[3])):
            np.add.at(lam, (si, rz[None, :], ry[None, :], rx[None, :]), r[:, it, :])
        if free_surface:                                   # vz[fs-1] = vz[fs]
            lz[:, fs] += lz[:, fs - 1]
            lz[:, fs - 1] = 0
        pn = hist_p[it]
        # adjoint of the velocity updates (they read p^{n+1})
        zs, ze = fs, Nz - 1
        for lam, kk, zr, yr, xr, axis in ((lx, k2, (zs, ze), (1, Ny - 1), (1, Nx - 2), 3),
                                          (ly, k3, (zs, ze), (1, Ny - 2), (1, Nx - 1), 2),
                                          (lz, k4, (fs, Nz - 2), (1, Ny - 1), (1, Nx - 1), 1)):
            R = (slice(None), slice(*zr), slice(*yr), slice(*xr))
            Rc = R[1:]

            def sh(d):     # the region shifted by d along this component's axis
                s = list(R)
                a, b = (zr, yr, xr)[axis - 1]
                s[axis] = slice(a + d, b + d)
                return tuple(s)
            gp = c1 * (pn[sh(1)] - pn[sh(0)]) + c2 * (pn[sh(2)] - pn[sh(-1)])
            g2[Rc] += (lam[R] * (-gp)).sum(axis=0)
            wv = a2[Rc] * lam[R]
            lp[sh(1)] += -c1 * wv
            lp[sh(0)] += c1 * wv
            lp[sh(2)] += -c2 * wv
            lp[sh(-1)] += c2 * wv
            lam[R] = (1 - kk[Rc]) * lam[R]
        if free_surface:                                   # p[fs-1] = -p[fs+1]
            lp[:, fs + 1] -= lp[:, fs - 1]
            lp[:, fs - 1] = 0
        gw[:, it] = dt * lp[np.arange(S), sz, sy, sx]      # adjoint of the source line
        # adjoint of the pressure update (it reads v^n)
        vxn, vyn, vzn = hist_v[it]
        R = (slice(None), slice(z0, z1), slice(y0, y1), slice(x0, x1))
        Rc = R[1:]
        dvx = (c1 * (vxn[:, z0:z1, y0:y1, x0:x1] - vxn[:, z0:z1, y0:y1, x0 - 1:x1 - 1]) +
               c2 * (vxn[:, z0:z1, y0:y1, x0 + 1:x1 + 1] - vxn[:, z0:z1, y0:y1, x0 - 2:x1 - 2]))
        dvy = (c1 * (vyn[:, z0:z1, y0:y1, x0:x1] - vyn[:, z0:z1, y0 - 1:y1 - 1, x0:x1]) +
               c2 * (vyn[:, z0:z1, y0 + 1:y1 + 1, x0:x1] - vyn[:, z0:z1, y0 - 2:y1 - 2, x0:x1]))
        dvz = (c1 * (vzn[:, z0:z1, y0:y1, x0:x1] - vzn[:, z0 - 1:z1 - 1, y0:y1, x0:x1]) +
               c2 * (vzn[:, z0 + 1:z1 + 1, y0:y1, x0:x1] - vzn[:, z0 - 2:z1 - 2, y0:y1, x0:x1]))
        g1[Rc] += (lp[R] * (-(dvx + dvy + dvz))).sum(axis=0)
        u = a1[Rc] * lp[R]
        for lam, axis in ((lx, 3), (ly, 2), (lz, 1)):
            def sh(d):
                s = list(R)
                a, b = ((z0, z1), (y0, y1), (x0, x1))[axis - 1]
                s[axis] = slice(a + d, b + d)
                return tuple(s)
            lam[sh(0)] += -c1 * u
            lam[sh(-1)] += c1 * u
            lam[sh(1)] += -c2 * u
            lam[sh(-2)] += c2 * u
        lp[R] = (1 - k1[Rc]) * lp[R]
    g_c = g1 * 2 * den * c * dt / dz
    g_den = g1 * c * c * dt / dz - g2 * dt / (den * den * dz)

    def fold(g):
        out = np.zeros((nz, ny, nx))
        iz = np.clip(np.arange(Nz) - nabc, 0, nz - 1)
        iy = np.clip(np.arange(Ny) - nabc, 0, ny - 1)
        ix = np.clip(np.arange(Nx) - nabc, 0, nx - 1)
        np.add.at(out, (iz[:, None, None], iy[None, :, None], ix[None, None, :]), g)
        return out
    if with_wavelet:
        return fold(g_c), fold(g_den), gw
    return fold(g_c), fold(g_den)
