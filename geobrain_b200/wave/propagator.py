"""AcousticPropagator: model + survey -> WaveResult, on the CUDA library.

Same constructor and forward() as
geobrain/physics/wave/propagators/acoustic.py:23-300:
  * the damping array is built once at construction from max(vp) at that
    moment (:121-148; vmax stays frozen afterwards, as in the reference);
  * forward() calls model.forward() (Gardner / clipping, :196), turns
    checkpointing off when no parameter requires grad (:199-202), selects
    one shot with shot_index (:205-216) and returns a WaveResult (:275).
Opt-in additions: fd_order (4 or 8) in the constructor; checkpoint_every,
snapshot_dtype, imaging_cache, imaging_dtype and want_energy in forward().
"""
from __future__ import annotations

from typing import Optional

import torch

from .boundary import create_boundary
from .kernel import acoustic_forward_kernel
from .kernel3d import acoustic_forward_kernel_3d
from .model import AbstractModel, AcousticModel, numpy2tensor
from .result import WaveResult
from .survey import Survey


class AbstractPropagator(torch.nn.Module):
    def __init__(self, model: AbstractModel, device: str = "cpu", dtype: torch.dtype = torch.float32) -> None:
        super().__init__()
        self.model = model
        self.device = device
        self.dtype = dtype
        self.ox, self.oz = model.ox, model.oz
        self.dx, self.dz = model.dx, model.dz
        self.nx, self.nz = model.nx, model.nz
        self.ny, self.dy, self.oy = model.ny, model.dy, model.oy
        self.abc_type = model.abc_type
        self.nabc = model.nabc
        self.free_surface = model.free_surface

    def forward(self, **kwargs):
        raise NotImplementedError

    def __repr__(self) -> str:
        return (f"{type(self).__name__}(\n  model={type(self.model).__name__},\n  grid=({self.nx}, {self.nz}),\n"
                f"  device='{self.device}'\n)")


class AcousticPropagator(AbstractPropagator):
    def __init__(self, model: AcousticModel, survey: Survey, device: str = "cpu",
                 dtype: torch.dtype = torch.float32, fd_order: int = 4) -> None:
        super().__init__(model, device, dtype)
        if not isinstance(model, AcousticModel):
            raise TypeError(f"Expected AcousticModel, got {type(model).__name__}")
        if not isinstance(survey, Survey):
            raise TypeError(f"Expected Survey, got {type(survey).__name__}")
        if model.ndim == 3 and fd_order != 4:
            raise ValueError("the 3-D acoustic kernel is 4th order")
        self.survey = survey
        self.nt, self.dt, self.f0 = survey.nt, survey.dt, survey.f0
        self.fd_order = fd_order
        self.damp = None
        self._init_boundary()
        self.source = survey.source
        src = self.source.get_loc()
        self.src_n = self.source.num
        self.wavelet = numpy2tensor(self.source.get_wavelet(), dtype).to(device)
        # locations are (x, z) in 2-D and (x, y, z) in 3-D (acoustic.py:90-116)
        self.src_x = numpy2tensor(src[:, 0], torch.long).to(device)
        self.src_z = numpy2tensor(src[:, -1], torch.long).to(device)
        if model.ndim == 3:
            self.src_y = numpy2tensor(src[:, 1], torch.long).to(device)
        self.receiver = survey.receiver
        rcv = self.receiver.get_loc()
        self.rcv_n = self.receiver.num
        self.rcv_x = numpy2tensor(rcv[:, 0], torch.long).to(device)
        self.rcv_z = numpy2tensor(rcv[:, -1], torch.long).to(device)
        if model.ndim == 3:
            self.rcv_y = numpy2tensor(rcv[:, 1], torch.long).to(device)
        self.receiver_masks = survey.receiver_masks

    def _init_boundary(self, vmax: Optional[float] = None) -> None:
        if vmax is None:
            vmax = float(self.model.vp.detach().cpu().max())
        extra = dict(ny=self.ny, dy=self.dy) if self.model.ndim == 3 else {}
        damp = create_boundary(self.abc_type, nx=self.nx, nz=self.nz, dx=self.dx, dz=self.dz, n_layers=self.nabc,
                               vmax=vmax, alpha=self.model.abc_alpha, free_surface=False, **extra)
        self.damp = numpy2tensor(damp, self.dtype).to(self.device)

    def forward(self, model: Optional[AcousticModel] = None, shot_index: Optional[int] = None,
                checkpoint_segments: int = 1, snapshot_every: int = 0, *, checkpoint_every: int = 0,
                snapshot_dtype: str = "fp32", want_energy: bool = True, imaging_cache="auto",
                imaging_dtype: str = "fp32", memory_budget: Optional[int] = None,
                absorbing: str = "damping") -> WaveResult:
        model = model if model is not None else self.model
        model.forward()
        if checkpoint_segments > 1 and not any(p.requires_grad for p in model.parameters()):
            checkpoint_segments = 1
        if shot_index is not None:
            sl = slice(shot_index, shot_index + 1)
            src_x, src_z, src_n, wavelet = self.src_x[sl], self.src_z[sl], 1, self.wavelet[sl]
        else:
            src_x, src_z, src_n, wavelet = self.src_x, self.src_z, self.src_n, self.wavelet
        if self.model.ndim == 3:
            if absorbing != "damping":
                raise NotImplementedError("3-D models use the damping layers (absorbing='damping')")
            src_y = self.src_y[sl] if shot_index is not None else self.src_y
            result = acoustic_forward_kernel_3d(
                nx=self.nx, ny=self.ny, nz=self.nz, dx=self.dx, dy=self.dy, dz=self.dz, nt=self.nt, dt=self.dt,
                nabc=self.nabc, free_surface=self.free_surface, src_x=src_x, src_y=src_y, src_z=src_z,
                src_n=src_n, src_v=wavelet, rcv_x=self.rcv_x, rcv_y=self.rcv_y, rcv_z=self.rcv_z,
                rcv_n=self.rcv_n, damp=self.damp, vp=model.vp, rho=model.rho,
                checkpoint_segments=checkpoint_segments, device=torch.device(self.device), dtype=self.dtype,
                imaging_cache="auto" if imaging_cache in ("auto", "all") else 0)
            return WaveResult.from_dict(result)
        result = acoustic_forward_kernel(
            nx=self.nx, nz=self.nz, dx=self.dx, dz=self.dz, nt=self.nt, dt=self.dt, nabc=self.nabc,
            free_surface=self.free_surface, src_x=src_x, src_z=src_z, src_n=src_n, src_v=wavelet,
            rcv_x=self.rcv_x, rcv_z=self.rcv_z, rcv_n=self.rcv_n, damp=self.damp, vp=model.vp, rho=model.rho,
            checkpoint_segments=checkpoint_segments, device=torch.device(self.device), dtype=self.dtype,
            snapshot_every=snapshot_every, fd_order=self.fd_order, checkpoint_every=checkpoint_every,
            snapshot_dtype=snapshot_dtype, want_energy=want_energy, imaging_cache=imaging_cache,
            imaging_dtype=imaging_dtype, memory_budget=memory_budget, absorbing=absorbing)
        return WaveResult.from_dict(result)

    def __call__(self, model: Optional[AcousticModel] = None, shot_index: Optional[int] = None,
                 checkpoint_segments: int = 1, snapshot_every: int = 0, **kw) -> WaveResult:
        return self.forward(model=model, shot_index=shot_index, checkpoint_segments=checkpoint_segments,
                            snapshot_every=snapshot_every, **kw)
