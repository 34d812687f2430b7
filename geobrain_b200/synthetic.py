"""Seeded synthetic velocity models and acquisitions for the benchmark
workloads (no public dataset is used; every model is generated here).

The reference's own geostatistics (FFT moving average) is isotropic in 2-D,
so the anisotropic Gaussian fields the workloads call for come from a
spectral filter of white noise: FFT of N(0, 1) noise times the square root of
the Fourier transform of the Gaussian covariance
exp(-(x/lx)^2 - (z/lz)^2), transformed back and normalised to unit standard
deviation.  All randomness is numpy PCG64 with the seed given.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np


def gaussian_field(nz: int, nx: int, dx: float, lz: float, lx: float, seed: int) -> np.ndarray:
    """Zero-mean, unit-variance stationary field with Gaussian covariance of
    correlation lengths lz (vertical) and lx (horizontal), in metres."""
    rng = np.random.default_rng(seed)
    pz, px = nz + int(4 * lz / dx) + 1, nx + int(4 * lx / dx) + 1   # pad against wrap-around
    noise = rng.standard_normal((pz, px))
    kz = np.fft.fftfreq(pz, d=dx) * 2 * np.pi
    kx = np.fft.rfftfreq(px, d=dx) * 2 * np.pi
    # spectrum of exp(-(x/l)^2) is proportional to exp(-(k l)^2 / 4)
    amp = np.exp(-((kz[:, None] * lz) ** 2 + (kx[None, :] * lx) ** 2) / 8.0)
    f = np.fft.irfft2(np.fft.rfft2(noise) * amp, s=(pz, px))[:nz, :nx]
    f -= f.mean()
    sd = f.std()
    return f / (sd if sd > 0 else 1.0)


def layered(nz: int, nx: int, rng: np.random.Generator, vtop: float = 1500.0, vbot: float = 3500.0,
            n_layers: int = 5, dv: float = 300.0) -> np.ndarray:
    """Linear depth gradient plus n_layers flat layers of random depth,
    thickness and +-dv velocity offset."""
    z = np.arange(nz, dtype=np.float64)[:, None]
    vp = vtop + (vbot - vtop) * z / max(nz - 1, 1) + np.zeros((nz, nx))
    for _ in range(n_layers):
        top = int(rng.integers(0, nz - 1))
        thick = int(rng.integers(2, max(3, nz // 4)))
        vp[top:top + thick, :] += rng.uniform(-dv, dv)
    return vp


def ricker(f0: float, dt: float, nt: int) -> np.ndarray:
    """Ricker wavelet of the reference's length rule, zero-padded to nt
    (un-integrated)."""
    nw = 2 * int(2.2 / f0 / dt / 2) + 1
    t = (np.arange(nw) - nw // 2) * dt
    arg = (np.pi * f0 * t) ** 2
    w = ((1.0 - 2.0 * arg) * np.exp(-arg)).astype(np.float32)
    out = np.zeros(nt, np.float32)
    out[:min(nt, nw)] = w[:nt]
    return out


@dataclass
class Workload:
    """One model with its acquisition."""
    name: str
    nz: int
    nx: int
    dx: float
    dt: float
    nt: int
    nabc: int
    fd_order: int
    vp: np.ndarray                      # model the gradient is taken at
    rho: np.ndarray
    src_x: np.ndarray
    src_z: np.ndarray
    rcv_x: np.ndarray
    rcv_z: np.ndarray
    wavelet: np.ndarray                 # (nt,)
    vp_true: Optional[np.ndarray] = None
    free_surface: bool = False
    extra: dict = field(default_factory=dict)

    @property
    def n_shots(self) -> int:
        return int(self.src_x.size)

    @property
    def cells(self) -> int:
        return (self.nz + 2 * self.nabc) * (self.nx + 2 * self.nabc)

    def cell_updates(self) -> int:
        """(shot, padded cell, step) units of one forward pass."""
        return self.n_shots * self.cells * self.nt


def plain_forward_100x200(seed: int = 0) -> Workload:
    """100 x 200, dx 10 m, dt 1 ms, 1000 steps, 4th order, 20-cell PML;
    1500 -> 3500 m/s depth gradient plus 5 flat layers (+-300 m/s), density
    2200; one 15 Hz Ricker at the surface centre, 200 surface receivers."""
    rng = np.random.default_rng(seed)
    nz, nx = 100, 200
    vp = layered(nz, nx, rng).astype(np.float32)
    return Workload("plain_forward_100x200", nz, nx, 10.0, 1e-3, 1000, 20, 4, vp,
                    np.full((nz, nx), 2200.0, np.float32), np.array([100]), np.array([1]),
                    np.arange(nx), np.ones(nx, dtype=np.int64), ricker(15.0, 1e-3, 1000))


def fwi_400x1200(seed: int = 0, nt: int = 3000, n_shots: int = 32) -> Workload:
    """400 x 1200, dx 10 m, dt 0.8 ms, 3000 steps, 8th order, 30-cell PML.
    True model: depth gradient (mean 2800) plus a Gaussian field (200 m
    horizontal / 50 m vertical correlation, std 250 m/s); the gradient is
    taken at a 400 m Gaussian smoothing of it.  32 evenly spaced 10 Hz Ricker
    shots at the surface, 1200 receivers, L2 trace misfit."""
    from scipy.ndimage import gaussian_filter
    nz, nx, dx = 400, 1200, 10.0
    z = np.arange(nz)[:, None] / (nz - 1)
    true = 2800.0 + 600.0 * (z - 0.5) + 250.0 * gaussian_field(nz, nx, dx, 50.0, 200.0, seed)
    true = np.clip(true, 1500.0, 4500.0).astype(np.float32)
    init = gaussian_filter(true.astype(np.float64), sigma=400.0 / dx, mode="nearest").astype(np.float32)
    sx = np.round(np.linspace(0, nx - 1, n_shots + 2)[1:-1]).astype(np.int64)
    return Workload("fwi_400x1200", nz, nx, dx, 8e-4, nt, 30, 8, init, np.full((nz, nx), 2200.0, np.float32),
                    sx, np.ones(n_shots, np.int64), np.arange(nx), np.ones(nx, dtype=np.int64),
                    ricker(10.0, 8e-4, nt), vp_true=true)


def ensemble_256x512(n_particles: int = 50, seed: int = 0, nt: int = 2000) -> List[Workload]:
    """50 particles of 256 x 512 (dx 10 m, dt 1 ms, 2000 steps, 8th order,
    20-cell PML), each an independent Gaussian field (150 m / 40 m, mean
    2500, std 200 m/s); 8 shots and 512 receivers each."""
    out = []
    nz, nx, dx = 256, 512, 10.0
    for p in range(n_particles):
        vp = np.clip(2500.0 + 200.0 * gaussian_field(nz, nx, dx, 40.0, 150.0, seed + 1000 + p), 1500, 4500)
        sx = np.round(np.linspace(0, nx - 1, 10)[1:-1]).astype(np.int64)
        out.append(Workload(f"particle_{p}", nz, nx, dx, 1e-3, nt, 20, 8, vp.astype(np.float32),
                            np.full((nz, nx), 2200.0, np.float32), sx, np.ones(8, np.int64), np.arange(nx),
                            np.ones(nx, dtype=np.int64), ricker(10.0, 1e-3, nt)))
    return out


def uneven_batch(n_models: int = 24, seed: int = 0, nt_scale: float = 1.0) -> List[Workload]:
    """24 models with sizes from {128x256, 256x512, 384x768, 512x1024}, step
    counts from {1000, 2000, 3000} and 4 to 16 shots; layered plus Gaussian
    fields clipped to 1500-4500 m/s; dx 10 m, dt 1 ms, 8th order, 20-cell PML."""
    rng = np.random.default_rng(seed)
    sizes = [(128, 256), (256, 512), (384, 768), (512, 1024)]
    out = []
    for m in range(n_models):
        nz, nx = sizes[int(rng.integers(0, 4))]
        nt = max(1, int(int(rng.choice([1000, 2000, 3000])) * nt_scale))
        ns = int(rng.integers(4, 17))
        vp = layered(nz, nx, rng, 1500.0, 4000.0) + 200.0 * gaussian_field(nz, nx, 10.0, 40.0, 150.0,
                                                                           seed + 2000 + m)
        vp = np.clip(vp, 1500.0, 4500.0).astype(np.float32)
        sx = np.round(np.linspace(0, nx - 1, ns + 2)[1:-1]).astype(np.int64)
        out.append(Workload(f"model_{m}", nz, nx, 10.0, 1e-3, nt, 20, 8, vp,
                            np.full((nz, nx), 2200.0, np.float32), sx, np.ones(ns, np.int64), np.arange(nx),
                            np.ones(nx, dtype=np.int64), ricker(10.0, 1e-3, nt)))
    return out


def large_1000x3000(seed: int = 0, nt: int = 8000) -> Workload:
    """1000 x 3000, dx 5 m, dt 0.4 ms, 8000 steps, 8th order, 40-cell PML,
    16 shots, 3000 receivers; layered model with a Gaussian perturbation of
    std 300 m/s."""
    rng = np.random.default_rng(seed)
    nz, nx, dx = 1000, 3000, 5.0
    vp = layered(nz, nx, rng, 1500.0, 4000.0) + 300.0 * gaussian_field(nz, nx, dx, 40.0, 150.0, seed + 3000)
    vp = np.clip(vp, 1500.0, 4500.0).astype(np.float32)
    sx = np.round(np.linspace(0, nx - 1, 18)[1:-1]).astype(np.int64)
    return Workload("large_1000x3000", nz, nx, dx, 4e-4, nt, 40, 8, vp, np.full((nz, nx), 2200.0, np.float32),
                    sx, np.ones(16, np.int64), np.arange(nx), np.ones(nx, dtype=np.int64), ricker(10.0, 4e-4, nt))


def cfl_number(vmax: float, dt: float, dx: float, fd_order: int) -> float:
    """Courant number of the staggered scheme in 2-D: vmax dt / dx * sum|c_k| * sqrt(2)."""
    c = {4: [9 / 8, 1 / 24], 8: [1225 / 1024, 245 / 3072, 49 / 5120, 5 / 7168]}[fd_order]
    return vmax * dt / dx * sum(c) * np.sqrt(2.0)
