"""Source wavelets (host side).

RickerWavelet / GaussianWavelet / create_wavelet keep the call signatures of
geobrain/physics/wave/wavelets/ricker.py:19-170 and wavelets/__init__.py:26-117:
an odd length nw = 2 int(L / f0 / dt / 2) + 1 centred on sample nw // 2, in
float32.  Only the two analytic pulses are provided; the band-pass
(Ormsby / Klauder) generators are not on the propagator path.
"""
from __future__ import annotations

import math
from typing import Optional, Tuple

import torch
from torch import Tensor


def _axis(length_factor: float, f0: float, dt: float, device) -> Tensor:
    nw = 2 * int(length_factor / f0 / dt / 2) + 1
    return (torch.arange(nw, device=device, dtype=torch.float32) - nw // 2) * dt


class WaveletGenerator(torch.nn.Module):
    def forward(self, f0: float, dt: float, device: Optional[str] = None) -> Tuple[Tensor, Tensor]:
        raise NotImplementedError


class RickerWavelet(WaveletGenerator):
    """w(t) = (1 - 2 (pi f0 t)^2) exp(-(pi f0 t)^2) on a symmetric axis."""

    def __init__(self, length_factor: float = 2.2):
        super().__init__()
        self.length_factor = length_factor

    def forward(self, f0, dt, device=None):
        f0 = f0.item() if isinstance(f0, Tensor) else f0
        dt = dt.item() if isinstance(dt, Tensor) else dt
        t = _axis(self.length_factor, f0, dt, device or "cpu")
        arg = math.pi * f0 * t
        return (1.0 - 2.0 * arg ** 2) * torch.exp(-arg ** 2), t

    def get_length(self, f0: float, dt: float) -> int:
        return 2 * int(self.length_factor / f0 / dt / 2) + 1


class GaussianWavelet(WaveletGenerator):
    """w(t) = exp(-4 f0^2 t^2)."""

    def __init__(self, length_factor: float = 2.0):
        super().__init__()
        self.length_factor = length_factor

    def forward(self, f0, dt, device=None):
        f0 = f0.item() if isinstance(f0, Tensor) else f0
        dt = dt.item() if isinstance(dt, Tensor) else dt
        t = _axis(self.length_factor, f0, dt, device or "cpu")
        return torch.exp(-4.0 * f0 ** 2 * t ** 2), t


def create_wavelet(wavelet_type: str, f0: float, dt: float, nt: Optional[int] = None, device: str = None,
                   **kwargs) -> Tuple[Tensor, Tensor]:
    kind = wavelet_type.lower()
    if kind in ("ricker", "mexican_hat"):
        gen = RickerWavelet()
    elif kind == "gaussian":
        gen = GaussianWavelet()
    elif kind in ("ormsby", "klauder"):
        raise NotImplementedError(f"'{kind}' wavelets are not on the propagator path")
    else:
        raise ValueError(f"Unknown wavelet type: '{wavelet_type}'. "
                         f"Choose from: 'ricker', 'gaussian', 'ormsby', 'klauder'")
    w, t = gen(f0, dt, device=device)
    if nt is not None:
        n = w.shape[0]
        if n < nt:
            extra = nt - n
            w = torch.cat([w, torch.zeros(extra, device=w.device)])
            t = torch.cat([t, t[-1] + dt * torch.arange(1, extra + 1, device=t.device)])
        else:
            w, t = w[:nt], t[:nt]
    return w, t
