"""3-D acoustic forward modelling with the reference's call signature.

``acoustic_forward_kernel_3d`` is a drop-in for
geobrain/physics/wave/kernels/acoustic_3d.py:303-476.  It takes the same
arguments (positions are unpadded grid indices; damp is the padded 3-D
array) and returns the same dict: traces p / vx / vy / vz (src_n, nt, rcv_n)
and energy maps forward_wavefield_{p,vx,vy,vz} (nz, ny, nx).  The CUDA
library (gb3_forward) computes them.  As in the reference, every derivative
is scaled by 1/dz.  The path is forward-only: a vp or rho that requires grad
raises.
"""
from __future__ import annotations

import ctypes

import torch
from torch import Tensor

from .. import _lib
from . import engine
from .kernel import _as_f32


def pad_model_3d(v: Tensor, pml: int, nz: int, ny: int, nx: int, device: torch.device = torch.device("cpu")) -> Tensor:
    """Edge-replicating pad of an (nz, ny, nx) model on all six faces
    (kernels/acoustic_2d.py:70-120).  The CUDA path pads inside its
    coefficient kernel; this host version is kept for API parity."""
    iz = torch.clamp(torch.arange(nz + 2 * pml, device=v.device) - pml, 0, nz - 1)
    iy = torch.clamp(torch.arange(ny + 2 * pml, device=v.device) - pml, 0, ny - 1)
    ix = torch.clamp(torch.arange(nx + 2 * pml, device=v.device) - pml, 0, nx - 1)
    return v[iz][:, iy][:, :, ix].to(device)


def acoustic_forward_kernel_3d(nx: int, ny: int, nz: int, dx: float, dy: float, dz: float, nt: int, dt: float,
                               nabc: int, free_surface: bool, src_x: Tensor, src_y: Tensor, src_z: Tensor,
                               src_n: int, src_v: Tensor, rcv_x: Tensor, rcv_y: Tensor, rcv_z: Tensor, rcv_n: int,
                               damp: Tensor, vp: Tensor, rho: Tensor, checkpoint_segments: int = 1,
                               device: torch.device = torch.device("cpu"), dtype: torch.dtype = torch.float32):
    device = torch.device(device)
    if device.type != "cuda":
        raise ValueError(f"geobrain_b200 runs on CUDA devices only (device={device})")
    if dtype != torch.float32:
        raise TypeError(f"geobrain_b200 computes in float32 (dtype={dtype})")
    if checkpoint_segments < 1:
        raise ValueError(f"checkpoint_segments must be >= 1, got {checkpoint_segments}")
    if torch.is_grad_enabled() and (getattr(vp, "requires_grad", False) or getattr(rho, "requires_grad", False)):
        raise NotImplementedError("the 3-D path of geobrain_b200 is forward-only (no gradient)")
    nx, ny, nz, nt, nabc, src_n, rcv_n = (int(v) for v in (nx, ny, nz, nt, nabc, src_n, rcv_n))
    pos = [engine._i64(a) for a in (src_x, src_y, src_z)]
    rpos = [engine._i64(a) for a in (rcv_x, rcv_y, rcv_z)]
    if any(p.size < src_n for p in pos) or any(p.size < rcv_n for p in rpos):
        raise ValueError("src_n / rcv_n exceed the position arrays")
    pos = [p[:src_n].copy() for p in pos]
    rpos = [p[:rcv_n].copy() for p in rpos]
    w = _as_f32(src_v, device, "src_v")
    if w.dim() == 1:
        w = w.unsqueeze(0).expand(src_n, -1)
    if tuple(w.shape) != (src_n, nt):
        raise ValueError(f"src_v must be (src_n, nt) = {(src_n, nt)} or (nt,), got {tuple(w.shape)}")
    w = w.contiguous()
    shape = (nz + 2 * nabc, ny + 2 * nabc, nx + 2 * nabc)
    damp_t = _as_f32(damp, device, "damp")
    if tuple(damp_t.shape) != shape:
        raise ValueError(f"damp must have shape {shape}, got {tuple(damp_t.shape)}")
    vp_t = _as_f32(vp.detach() if torch.is_tensor(vp) else vp, device, "vp")
    rho_t = _as_f32(rho.detach() if torch.is_tensor(rho) else rho, device, "rho")
    for name, t in (("vp", vp_t), ("rho", rho_t)):
        if tuple(t.shape) != (nz, ny, nx):
            raise ValueError(f"{name} must have shape {(nz, ny, nx)}, got {tuple(t.shape)}")
    desc = _lib.Desc3(nz, ny, nx, nabc, nt, src_n, rcv_n, int(bool(free_surface)), float(dt), float(dx), float(dy),
                      float(dz))
    L = _lib.load()
    ws = engine.workspace(int(L.gb3_workspace_bytes(ctypes.byref(desc))), device)
    f32 = dict(device=device, dtype=torch.float32)
    tr = [torch.empty((src_n, nt, rcv_n), **f32) for _ in range(4)]
    en = [torch.empty((nz, ny, nx), **f32) for _ in range(4)]
    with torch.cuda.device(device):
        rc = L.gb3_forward(ctypes.byref(desc), *[p.ctypes.data for p in pos], *[p.ctypes.data for p in rpos],
                           vp_t.data_ptr(), rho_t.data_ptr(), damp_t.data_ptr(), w.data_ptr(),
                           *[t.data_ptr() for t in tr], *[e.data_ptr() for e in en], ws.data_ptr(), ws.numel(),
                           engine.stream_handle(device))
    if rc == _lib.GB_E_ARG:
        raise ValueError(L.gb_last_error().decode())
    _lib.check(rc)
    keys = ("p", "vx", "vy", "vz")
    out = {k: t for k, t in zip(keys, tr)}
    out.update({f"forward_wavefield_{k}": e for k, e in zip(keys, en)})
    return out
