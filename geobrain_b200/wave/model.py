"""Velocity models: AbstractModel and AcousticModel.

API of geobrain/physics/wave/core/base.py:33-293 (AbstractModel) and
geobrain/physics/wave/models/acoustic.py:20-199 (AcousticModel): vp and rho
are nn.Parameters; forward() applies Gardner's density update
(rho = 310 vp^0.25, outside autograd, keeping a water-layer mask) when
auto_update_rho and not rho_grad, then clips to the bounds.
"""
from __future__ import annotations

from typing import Dict, Optional, Tuple, Union

import numpy as np
import torch
import torch.nn as nn

from .config import BoundaryConfig, GridConfig

UNITS = {"vp": "m/s", "vs": "m/s", "rho": "kg/m³", "lam": "Pa", "mu": "Pa", "eps": "", "gamma": "", "delta": ""}


def numpy2tensor(a, dtype: torch.dtype = torch.float32) -> torch.Tensor:
    if torch.is_tensor(a):
        return a.to(dtype)
    return torch.tensor(np.asarray(a), dtype=dtype)


class AbstractModel(nn.Module):
    def __init__(self, grid: GridConfig, boundary: BoundaryConfig, device: str = "cpu",
                 dtype: torch.dtype = torch.float32) -> None:
        super().__init__()
        self.grid = grid
        self.ox, self.oz = grid.ox, grid.oz
        self.dx, self.dz = grid.dx, grid.dz
        self.nx, self.nz = grid.nx, grid.nz
        self.ny, self.dy, self.oy = grid.ny, grid.dy, grid.oy
        self.boundary = boundary
        self.free_surface = boundary.free_surface
        self.abc_type = boundary.type
        self.abc_alpha = boundary.alpha
        self.nabc = boundary.n_layers
        self.device = device
        self.dtype = dtype
        self.x, self.z, self.y = grid.x, grid.z, grid.y
        self.pars: list = []
        self.requires_grad: Dict[str, bool] = {}
        self.lower_bound: Dict[str, Optional[float]] = {}
        self.upper_bound: Dict[str, Optional[float]] = {}

    @property
    def ndim(self) -> int:
        return self.grid.ndim

    @property
    def shape(self) -> tuple:
        return self.grid.shape

    def __repr__(self) -> str:
        lines = [f"{type(self).__name__} with parameters {self.pars}:"]
        for par in self.pars:
            m = self.get_model(par)
            lines.append(f"  {par:4s}: {m.min():8.2f} - {m.max():8.2f} {UNITS.get(par, ''):6s}, "
                         f"grad={self.requires_grad.get(par, False)}, "
                         f"bounds=[{self.lower_bound.get(par)}, {self.upper_bound.get(par)}]")
        lines.append(f"  Grid: {self.nx} x {self.nz}, dx={self.dx:.2f}m")
        lines.append(f"  Boundary: {self.abc_type}, {self.nabc} layers")
        lines.append(f"  Free surface: {self.free_surface}")
        return "\n".join(lines) + "\n"

    def forward(self) -> None:
        raise NotImplementedError

    def get_model(self, par: str) -> np.ndarray:
        if par not in self.pars:
            raise ValueError(f"Parameter '{par}' not in model. Available: {self.pars}")
        data = getattr(self, par)
        return data.detach().cpu().numpy().copy() if torch.is_tensor(data) else np.array(data)

    def set_model(self, par: str, model: Union[np.ndarray, torch.Tensor]) -> None:
        if par not in self.pars:
            raise ValueError(f"Parameter '{par}' not in model. Available: {self.pars}")
        if tuple(model.shape) != tuple(self.shape):
            raise ValueError(f"Shape mismatch: expected {self.shape}, got {model.shape}")
        t = model.to(dtype=self.dtype, device=self.device) if torch.is_tensor(model) else \
            torch.tensor(model, dtype=self.dtype, device=self.device)
        setattr(self, par, nn.Parameter(t, requires_grad=self.requires_grad.get(par, False)))

    def get_grad(self, par: str) -> np.ndarray:
        if par not in self.pars:
            raise ValueError(f"Parameter '{par}' not in model")
        m = getattr(self, par)
        return np.zeros(self.shape) if m.grad is None else m.grad.detach().cpu().numpy()

    def get_bound(self, par: str) -> Tuple[Optional[float], Optional[float]]:
        if par not in self.pars:
            raise ValueError(f"Parameter '{par}' not in model")
        return self.lower_bound.get(par), self.upper_bound.get(par)

    def clip_params(self) -> None:
        for par in self.pars:
            lb, ub = self.lower_bound.get(par), self.upper_bound.get(par)
            if lb is not None or ub is not None:
                getattr(self, par).data.clamp_(lb, ub)

    def save(self, filename: str) -> None:
        data = dict(ox=self.ox, oz=self.oz, dx=self.dx, dz=self.dz, nx=self.nx, nz=self.nz, ndim=self.ndim,
                    free_surface=self.free_surface, abc_type=self.abc_type, nabc=self.nabc)
        for par in self.pars:
            data[par] = self.get_model(par)
            data[f"{par}_bound"] = self.get_bound(par)
            data[f"{par}_grad"] = self.requires_grad.get(par, False)
        np.savez(filename, **data)


class AcousticModel(AbstractModel):
    def __init__(self, grid: GridConfig, boundary: BoundaryConfig, vp, rho,
                 vp_bound: Optional[Tuple[float, float]] = None, rho_bound: Optional[Tuple[float, float]] = None,
                 vp_grad: bool = False, rho_grad: bool = False, auto_update_rho: bool = True,
                 water_layer_mask=None, device: str = "cpu", dtype: torch.dtype = torch.float32) -> None:
        super().__init__(grid, boundary, device, dtype)
        self.pars = ["vp", "rho"]
        self.vp_grad, self.rho_grad = vp_grad, rho_grad
        self.requires_grad["vp"], self.requires_grad["rho"] = vp_grad, rho_grad
        self.auto_update_rho = auto_update_rho
        self._vp_init = vp.copy() if isinstance(vp, np.ndarray) else vp.clone()
        self._rho_init = rho.copy() if isinstance(rho, np.ndarray) else rho.clone()
        self._init_parameters(vp, rho)
        self.lower_bound["vp"], self.upper_bound["vp"] = vp_bound if vp_bound else (None, None)
        self.lower_bound["rho"], self.upper_bound["rho"] = rho_bound if rho_bound else (None, None)
        self.water_layer_mask = None if water_layer_mask is None else \
            numpy2tensor(water_layer_mask, torch.bool).to(device)
        self._validate()

    def _init_parameters(self, vp, rho) -> None:
        self.vp = nn.Parameter(numpy2tensor(vp, self.dtype).to(self.device), requires_grad=self.vp_grad)
        self.rho = nn.Parameter(numpy2tensor(rho, self.dtype).to(self.device), requires_grad=self.rho_grad)

    def _validate(self) -> None:
        for par in self.pars:
            lb, ub = self.lower_bound.get(par), self.upper_bound.get(par)
            if lb is not None and ub is not None and lb >= ub:
                raise ValueError(f"Invalid bounds for {par}: lower={lb} >= upper={ub}")
        for par in self.pars:
            if tuple(getattr(self, par).shape) != tuple(self.shape):
                raise ValueError(f"Shape mismatch for {par}: expected {self.shape}, "
                                 f"got {tuple(getattr(self, par).shape)}")

    def set_rho_empirical(self) -> None:
        """Gardner's relation rho = 310 vp^0.25 (water-layer cells keep their density)."""
        with torch.no_grad():
            vp = self.vp.detach().cpu().numpy()
            rho = 310.0 * np.power(vp, 0.25)
            if self.water_layer_mask is not None:
                mask = self.water_layer_mask.cpu().numpy()
                rho[mask] = self.rho.detach().cpu().numpy()[mask]
            self.rho = nn.Parameter(numpy2tensor(rho, self.dtype).to(self.device), requires_grad=self.rho_grad)

    def forward(self) -> None:
        if self.auto_update_rho and not self.rho_grad:
            self.set_rho_empirical()
        self.clip_params()

    def reset(self) -> None:
        self._init_parameters(self._vp_init, self._rho_init)
