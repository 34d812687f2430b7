"""WaveResult: the propagator's output container (dict-compatible).

Same fields and dict-style access as geobrain/physics/wave/core/result.py:17-119.
"""
from __future__ import annotations

from dataclasses import dataclass, fields
from typing import Optional

from torch import Tensor


@dataclass
class WaveResult:
    p: Tensor
    vx: Tensor
    vz: Tensor
    forward_wavefield_p: Tensor
    forward_wavefield_vx: Tensor
    forward_wavefield_vz: Tensor
    vy: Optional[Tensor] = None
    forward_wavefield_vy: Optional[Tensor] = None
    snapshots: Optional[Tensor] = None

    def __getitem__(self, key: str) -> Tensor:
        if key not in {f.name for f in fields(self)}:
            raise KeyError(key)
        return getattr(self, key)

    def __contains__(self, key: str) -> bool:
        return getattr(self, key, None) is not None

    def keys(self):
        return [f.name for f in fields(self) if getattr(self, f.name) is not None]

    def values(self):
        return [getattr(self, k) for k in self.keys()]

    def items(self):
        return [(k, getattr(self, k)) for k in self.keys()]

    @classmethod
    def from_dict(cls, d: dict) -> "WaveResult":
        return cls(p=d["p"], vx=d["vx"], vz=d["vz"], forward_wavefield_p=d["forward_wavefield_p"],
                   forward_wavefield_vx=d["forward_wavefield_vx"], forward_wavefield_vz=d["forward_wavefield_vz"],
                   vy=d.get("vy"), forward_wavefield_vy=d.get("forward_wavefield_vy"),
                   snapshots=d.get("snapshots"))

    @property
    def ndim(self) -> int:
        return 2 if self.vy is None else 3

    @property
    def n_shots(self) -> int:
        return self.p.shape[0]

    @property
    def nt(self) -> int:
        return self.p.shape[1]

    @property
    def n_receivers(self) -> int:
        return self.p.shape[2]
