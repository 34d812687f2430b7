"""CPU oracle of the CPML absorbing option of the 2-D forward, in NumPy.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA
CPML path; the product package never imports it.

The reference has no CPML: this restates the scheme this library defines
for it (gb_plan_set_absorbing in include/geobrain_b200.h) on top of the
reference's staggered leapfrog (geobrain/physics/wave/kernels/acoustic_2d.py
:211-285, generalised to half-width R).  Per axis a quadratic profile
d = d0 (depth / nabc)^2, d0 = -3 vmax ln(1e-6) / (2 nabc dx), on both sides
(none above a free surface), b = exp(-d dt), a = b - 1, at integer and half
points; every derivative g of an update becomes g + psi with
psi' = b psi + a g; no damping terms.  Float64, whole-array operations, for
small grids.  forward_torch restates it in torch for the gradient oracle.
"""
from __future__ import annotations

import math

import numpy as np


def fd_coefficients(half: int) -> np.ndarray:
    if half == 2:
        return np.array([9.0 / 8.0, -1.0 / 24.0])
    if half == 4:
        return np.array([1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0, -5.0 / 7168.0])
    raise ValueError("half must be 2 or 4")


def profiles(N: int, nabc: int, dx: float, dt: float, vmax: float, lo: bool):
    """(b, a) at integer points and (b, a) at half points of one axis."""
    d0 = -3.0 * vmax * math.log(1e-6) / (2.0 * nabc * dx)

    def one(c):
        r = 0.0
        if lo and c < nabc:
            r = (nabc - c) / nabc
        elif c > N - 1 - nabc:
            r = (c - (N - 1 - nabc)) / nabc
        r = min(r, 1.0)
        b = math.exp(-d0 * r * r * dt)
        return b, b - 1.0
    bi, ai = zip(*[one(i) for i in range(N)])
    bh, ah = zip(*[one(i + 0.5) for i in range(N)])
    return np.array(bi), np.array(ai), np.array(bh), np.array(ah)


def forward(*, nz, nx, dz, nt, dt, nabc, free_surface, src_x, src_z, src_v, rcv_x, rcv_z, vp, rho, half=4,
            vmax=None):
    c = np.pad(np.asarray(vp, np.float64), nabc, mode="edge")
    den = np.pad(np.asarray(rho, np.float64), nabc, mode="edge")
    Nz, Nx = nz + 2 * nabc, nx + 2 * nabc
    R = half
    cf = fd_coefficients(R)
    fs = nabc if free_surface else 1
    a1 = den * c * c * dt / dz
    a2 = dt / (den * dz)
    vmax = float(np.max(vp)) if vmax is None else float(vmax)
    bzi, azi, bzh, azh = profiles(Nz, nabc, dz, dt, vmax, not free_surface)
    bxi, axi, bxh, axh = profiles(Nx, nabc, dz, dt, vmax, True)
    S = len(src_x)
    sx, sz = np.asarray(src_x) + nabc, np.asarray(src_z) + nabc
    rx, rz = np.asarray(rcv_x) + nabc, np.asarray(rcv_z) + nabc
    w = np.asarray(src_v, np.float64)
    p = np.zeros((S, Nz, Nx))
    vx = np.zeros_like(p)
    vz = np.zeros_like(p)
    ppx, ppz, pvx, pvz = (np.zeros_like(p) for _ in range(4))
    tr = {k: np.zeros((S, nt, len(rx))) for k in ("p", "vx", "vz")}
    en = {k: np.zeros((nz, nx)) for k in ("p", "vx", "vz")}
    pr0, pr1, pc0, pc1 = max(fs + 1, R), Nz - 1 - R, R, Nx - 1 - R
    xr0, xr1, xc0, xc1 = fs, Nz - 2, R - 1, Nx - 1 - R
    zr0, zr1, zc0, zc1 = max(fs, R - 1), Nz - 1 - R, 1, Nx - 2
    for it in range(nt):
        I, J = slice(pr0, pr1 + 1), slice(pc0, pc1 + 1)
        Dx = sum(cf[k] * (vx[:, I, pc0 + k:pc1 + 1 + k] - vx[:, I, pc0 - 1 - k:pc1 - k]) for k in range(R))
        Dz = sum(cf[k] * (vz[:, pr0 + k:pr1 + 1 + k, J] - vz[:, pr0 - 1 - k:pr1 - k, J]) for k in range(R))
        ppx[:, I, J] = bxi[None, None, J] * ppx[:, I, J] + axi[None, None, J] * Dx
        ppz[:, I, J] = bzi[None, I, None] * ppz[:, I, J] + azi[None, I, None] * Dz
        p[:, I, J] -= a1[I, J] * ((Dx + ppx[:, I, J]) + (Dz + ppz[:, I, J]))
        p[np.arange(S), sz, sx] += dt * w[:, it]
        if free_surface:
            p[:, fs - 1] = -p[:, fs + 1]
        I, J = slice(xr0, xr1 + 1), slice(xc0, xc1 + 1)
        Gx = sum(cf[k] * (p[:, I, xc0 + 1 + k:xc1 + 2 + k] - p[:, I, xc0 - k:xc1 + 1 - k]) for k in range(R))
        pvx[:, I, J] = bxh[None, None, J] * pvx[:, I, J] + axh[None, None, J] * Gx
        vx[:, I, J] -= a2[I, J] * (Gx + pvx[:, I, J])
        I, J = slice(zr0, zr1 + 1), slice(zc0, zc1 + 1)
        Gz = sum(cf[k] * (p[:, zr0 + 1 + k:zr1 + 2 + k, J] - p[:, zr0 - k:zr1 + 1 - k, J]) for k in range(R))
        pvz[:, I, J] = bzh[None, I, None] * pvz[:, I, J] + azh[None, I, None] * Gz
        vz[:, I, J] -= a2[I, J] * (Gz + pvz[:, I, J])
        if free_surface:
            vz[:, fs - 1] = vz[:, fs]
        for k, f in (("p", p), ("vx", vx), ("vz", vz)):
            tr[k][:, it, :] = f[:, rz, rx]
            en[k] += (f * f).sum(axis=0)[nabc:nabc + nz, nabc:nabc + nx]
    out = dict(tr)
    out.update({f"forward_wavefield_{k}": v for k, v in en.items()})
    return out


def forward_torch(*, nz, nx, dz, nt, dt, nabc, free_surface, src_x, src_z, src_v, rcv_x, rcv_z, vp, rho, half=4,
                  vmax):
    """The same scheme in float64 torch, written functionally (masks and
    shifts, no in-place updates) so that autograd through it is the exact
    discrete adjoint: the gradient oracle of the CPML option.  vp and rho are
    (nz, nx) float64 tensors (they may require grad); vmax is a constant.
    Returns the (S, nt, R) traces of p, vx and vz."""
    import torch
    import torch.nn.functional as F
    R = half
    cf = fd_coefficients(R)
    Nz, Nx = nz + 2 * nabc, nx + 2 * nabc
    fs = nabc if free_surface else 1
    c = F.pad(vp[None, None], (nabc,) * 4, mode="replicate")[0, 0]
    den = F.pad(rho[None, None], (nabc,) * 4, mode="replicate")[0, 0]
    a1 = den * c * c * dt / dz
    a2 = dt / (den * dz)
    tt = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.float64)
    bzi, azi, bzh, azh = (tt(v)[:, None] for v in profiles(Nz, nabc, dz, dt, vmax, not free_surface))
    bxi, axi, bxh, axh = (tt(v)[None, :] for v in profiles(Nx, nabc, dz, dt, vmax, True))

    def box(r0, r1, c0, c1):
        m = torch.zeros(Nz, Nx, dtype=torch.float64)
        m[r0:r1 + 1, c0:c1 + 1] = 1.0
        return m
    Mp = box(max(fs + 1, R), Nz - 1 - R, R, Nx - 1 - R)
    Mvx = box(fs, Nz - 2, R - 1, Nx - 1 - R)
    Mvz = box(max(fs, R - 1), Nz - 1 - R, 1, Nx - 2)

    def shift(f, di, dj):
        """g[..., i, j] = f[..., i + di, j + dj], zero outside."""
        P = R + 2
        g = F.pad(f, (P, P, P, P))
        return g[..., P + di:P + di + Nz, P + dj:P + dj + Nx]

    S = len(src_x)
    sx, sz = np.asarray(src_x) + nabc, np.asarray(src_z) + nabc
    rx, rz = torch.as_tensor(np.asarray(rcv_x) + nabc), torch.as_tensor(np.asarray(rcv_z) + nabc)
    onehot = torch.zeros(S, Nz, Nx, dtype=torch.float64)
    onehot[torch.arange(S), torch.as_tensor(sz), torch.as_tensor(sx)] = 1.0
    w = src_v if torch.is_tensor(src_v) else tt(src_v)
    zero = torch.zeros(S, Nz, Nx, dtype=torch.float64)
    p, vx, vz, ppx, ppz, pvx, pvz = (zero,) * 7
    tr = {"p": [], "vx": [], "vz": []}
    for it in range(nt):
        Dx = sum(cf[k] * (shift(vx, 0, k) - shift(vx, 0, -1 - k)) for k in range(R))
        Dz = sum(cf[k] * (shift(vz, k, 0) - shift(vz, -1 - k, 0)) for k in range(R))
        ppx = Mp * (bxi * ppx + axi * Dx) + (1 - Mp) * ppx
        ppz = Mp * (bzi * ppz + azi * Dz) + (1 - Mp) * ppz
        p = p - Mp * a1 * ((Dx + ppx) + (Dz + ppz))
        p = p + dt * w[:, it, None, None] * onehot
        if free_surface:
            p = torch.cat([p[:, :fs - 1], -p[:, fs + 1:fs + 2], p[:, fs:]], dim=1)
        Gx = sum(cf[k] * (shift(p, 0, 1 + k) - shift(p, 0, -k)) for k in range(R))
        pvx = Mvx * (bxh * pvx + axh * Gx) + (1 - Mvx) * pvx
        vx = vx - Mvx * a2 * (Gx + pvx)
        Gz = sum(cf[k] * (shift(p, 1 + k, 0) - shift(p, -k, 0)) for k in range(R))
        pvz = Mvz * (bzh * pvz + azh * Gz) + (1 - Mvz) * pvz
        vz = vz - Mvz * a2 * (Gz + pvz)
        if free_surface:
            vz = torch.cat([vz[:, :fs - 1], vz[:, fs:fs + 1], vz[:, fs:]], dim=1)
        for k, f in (("p", p), ("vx", vx), ("vz", vz)):
            tr[k].append(f[:, rz, rx])
    return {k: torch.stack(v, dim=1) for k, v in tr.items()}


def gradient(*, res_p=None, res_vx=None, res_vz=None, vp, rho, src_v, with_wavelet=False, **kw):
    """dL/dvp and dL/drho (and, with_wavelet, dL/dsrc_v) of L = sum(res_p *
    p) + sum(res_vx * vx) + sum(res_vz * vz) over the traces, by float64
    autograd through forward_torch (res_* are (S, nt, R) weights, any may be
    None)."""
    import torch
    v = torch.tensor(np.asarray(vp, np.float64), requires_grad=True)
    r = torch.tensor(np.asarray(rho, np.float64), requires_grad=True)
    w = torch.tensor(np.asarray(src_v, np.float64), requires_grad=with_wavelet)
    tr = forward_torch(vp=v, rho=r, src_v=w, **kw)
    loss = sum((torch.as_tensor(np.asarray(x, np.float64)) * tr[k]).sum()
               for k, x in (("p", res_p), ("vx", res_vx), ("vz", res_vz)) if x is not None)
    loss.backward()
    if with_wavelet:
        return v.grad.numpy(), r.grad.numpy(), w.grad.numpy()
    return v.grad.numpy(), r.grad.numpy()
