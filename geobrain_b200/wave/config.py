"""Simulation configuration dataclasses.

Same names, fields, defaults and validation errors as
geobrain/physics/wave/core/config.py (GridConfig :17-127, BoundaryConfig
:130-164, TimeConfig :167-206, WaveletConfig :209-237, SolverConfig
:240-296).  SolverConfig.fd_order additionally selects the stencil of the
CUDA propagator here (4 or 8; the reference validates the field but never
reads it).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Literal, Optional, Tuple

import numpy as np
import torch


@dataclass
class GridConfig:
    """Regular grid: nx, nz points at spacing dx == dz (dy, ny for 3-D)."""

    nx: int
    nz: int
    dx: float
    dz: float
    ox: float = 0.0
    oz: float = 0.0
    ny: Optional[int] = None
    dy: Optional[float] = None
    oy: float = 0.0

    def __post_init__(self):
        if self.nx <= 0 or self.nz <= 0:
            raise ValueError(f"Grid dimensions must be positive: nx={self.nx}, nz={self.nz}")
        if self.dx <= 0 or self.dz <= 0:
            raise ValueError(f"Grid spacing must be positive: dx={self.dx}, dz={self.dz}")
        if self.dx != self.dz:
            raise ValueError(f"Grid spacing must be equal: dx={self.dx}, dz={self.dz}")
        if (self.ny is None) != (self.dy is None):
            raise ValueError("ny and dy must both be provided for 3-D grids")
        if self.ny is not None:
            if self.ny <= 0:
                raise ValueError(f"ny must be positive: {self.ny}")
            if self.dy <= 0:
                raise ValueError(f"dy must be positive: {self.dy}")
            if self.dy != self.dx:
                raise ValueError(f"Grid spacing must be equal: dx={self.dx}, dy={self.dy}")

    @property
    def ndim(self) -> int:
        return 2 if self.ny is None else 3

    @property
    def shape(self) -> tuple:
        return (self.nz, self.nx) if self.ny is None else (self.nz, self.ny, self.nx)

    @property
    def x(self) -> np.ndarray:
        return self.ox + self.dx * np.arange(self.nx)

    @property
    def z(self) -> np.ndarray:
        return self.oz + self.dz * np.arange(self.nz)

    @property
    def y(self) -> Optional[np.ndarray]:
        return None if self.ny is None else self.oy + self.dy * np.arange(self.ny)

    @property
    def extent(self) -> Tuple[float, float, float, float]:
        return (self.ox, self.ox + (self.nx - 1) * self.dx, self.oz + (self.nz - 1) * self.dz, self.oz)


@dataclass
class BoundaryConfig:
    """Absorbing boundary: type ('pml' on this path), layer count, free surface."""

    type: Literal["pml", "gerjan", "sincos"] = "pml"
    n_layers: int = 20
    free_surface: bool = False
    alpha: float = 0.0053

    def __post_init__(self):
        self.type = self.type.lower()
        if self.type not in ("pml", "gerjan", "sincos"):
            raise ValueError(f"Unknown boundary type: '{self.type}'. Choose from: 'pml', 'gerjan', 'sincos'")
        if self.n_layers <= 0:
            raise ValueError(f"Number of layers must be positive: {self.n_layers}")


@dataclass
class TimeConfig:
    nt: int
    dt: float
    t0: float = 0.0

    def __post_init__(self):
        if self.nt <= 0:
            raise ValueError(f"Number of time steps must be positive: {self.nt}")
        if self.dt <= 0:
            raise ValueError(f"Time step must be positive: {self.dt}")

    @property
    def duration(self) -> float:
        return self.nt * self.dt

    @property
    def t(self) -> np.ndarray:
        return self.t0 + self.dt * np.arange(self.nt)


@dataclass
class WaveletConfig:
    f0: float
    type: Literal["ricker", "gaussian", "ormsby", "klauder"] = "ricker"
    amp: float = 1.0
    delay: Optional[float] = None

    def __post_init__(self):
        self.type = self.type.lower()
        if self.f0 <= 0:
            raise ValueError(f"Frequency must be positive: {self.f0}")
        if self.delay is None:
            self.delay = 1.2 / self.f0


@dataclass
class SolverConfig:
    fd_order: int = 4
    device: str = "cpu"
    dtype: str = "float32"
    checkpoint_segments: int = 1

    def __post_init__(self):
        if self.fd_order not in (4, 6, 8, 10):
            raise ValueError(f"FD order must be 4, 6, 8, or 10, got {self.fd_order}")
        if self.device not in ("cpu", "cuda") and not self.device.startswith("cuda:"):
            raise ValueError(f"Unknown device: '{self.device}'")
        if self.dtype not in ("float32", "float64"):
            raise ValueError(f"Unknown dtype: '{self.dtype}'")
        if self.checkpoint_segments < 1:
            raise ValueError(f"Checkpoint segments must be >= 1, got {self.checkpoint_segments}")

    @property
    def torch_device(self) -> torch.device:
        return torch.device(self.device)

    @property
    def torch_dtype(self) -> torch.dtype:
        return torch.float64 if self.dtype == "float64" else torch.float32
