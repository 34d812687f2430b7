"""Kernel-level entry points with the reference's call signatures.

``acoustic_forward_kernel`` is a drop-in for
geobrain/physics/wave/kernels/acoustic_2d.py:294-501: same positional and
keyword arguments, same output dict (p/vx/vz traces (src_n, nt, rcv_n),
forward_wavefield_{p,vx,vz} (nz, nx), and 'snapshots' (n, nz, nx) on the CPU
when snapshot_every > 0), computed by the CUDA library.  When vp or rho
requires grad, the traces are differentiable through the hand-written
adjoint (engine.AcousticFunction); the energy maps are detached, as in the
reference.

Additions, all keyword-only with defaults that keep the reference's
behaviour: fd_order (4 or 8); checkpoint_every, snapshot_dtype ('fp32';
'fp24', 3 bytes, gradient error about 1e-5; 'fp16' and 'bf16', 2 bytes with
one scale per snapshot field, about 6e-4 and 5e-3), imaging_cache ('auto', 'all', a byte budget, or 0) and
imaging_dtype ('fp32'; 'fp24', 3 bytes, gradient error about 1e-5; 'bf16',
2 bytes, about 3e-3: more cached steps skip the recompute) for the
gradient's memory, and memory_budget (bytes the gradient's store and
workspaces may take, for the 'auto' cache); absorbing ('damping', the
reference's PML driven by damp, or 'cpml': memory-variable convolutional
PML layers, damp unused; its gradient keeps every step's imaging fields,
imaging_cache='all'); want_energy (skip the energy
sums); autotune (on the
first call for a geometry, time the launch configurations and keep the
fastest; GEOBRAIN_B200_AUTOTUNE=1 turns it on by default).
"""
from __future__ import annotations

import os
from typing import Optional

import torch
from torch import Tensor

from . import engine


def pad_model(v: Tensor, pml: int, nz: int, nx: int, device: torch.device = torch.device("cpu")) -> Tensor:
    """Edge-replicating pad of an (nz, nx) model to (nz + 2 pml, nx + 2 pml)
    (acoustic_2d.py:18-66).  The CUDA path pads inside its coefficient kernel;
    this host version is kept for API parity."""
    iz = torch.clamp(torch.arange(nz + 2 * pml, device=v.device) - pml, 0, nz - 1)
    ix = torch.clamp(torch.arange(nx + 2 * pml, device=v.device) - pml, 0, nx - 1)
    return v[iz][:, ix].to(device)


def _as_f32(t, device, name):
    if not torch.is_tensor(t):
        t = torch.as_tensor(t)
    if t.dtype not in (torch.float32, torch.float64, torch.float16, torch.bfloat16):
        raise TypeError(f"{name} must be a floating tensor")
    return t.to(device=device, dtype=torch.float32).contiguous()


def acoustic_forward_kernel(nx: int, nz: int, dx: float, dz: float, nt: int, dt: float, nabc: int,
                            free_surface: bool, src_x: Tensor, src_z: Tensor, src_n: int, src_v: Tensor,
                            rcv_x: Tensor, rcv_z: Tensor, rcv_n: int, damp: Tensor, vp: Tensor, rho: Tensor,
                            checkpoint_segments: int = 1, device: torch.device = torch.device("cpu"),
                            dtype: torch.dtype = torch.float32, snapshot_every: int = 0, *,
                            fd_order: int = 4, checkpoint_every: int = 0, snapshot_dtype: str = "fp32",
                            want_energy: bool = True, imaging_cache="auto", imaging_dtype: str = "fp32",
                            autotune: Optional[bool] = None, memory_budget: Optional[int] = None,
                            absorbing: str = "damping"):
    device = torch.device(device)
    if device.type != "cuda":
        raise ValueError(f"geobrain_b200 runs on CUDA devices only (device={device})")
    if dtype != torch.float32:
        raise TypeError(f"geobrain_b200 computes in float32 (dtype={dtype})")
    if float(dx) != float(dz):
        raise ValueError(f"Grid spacing must be equal: dx={dx}, dz={dz}")
    if fd_order not in engine.FD_ORDERS:
        raise ValueError(f"fd_order must be one of {sorted(engine.FD_ORDERS)}, got {fd_order}")
    if checkpoint_segments < 1:
        raise ValueError(f"checkpoint_segments must be >= 1, got {checkpoint_segments}")
    src_n, rcv_n = int(src_n), int(rcv_n)
    geo = engine.Geometry(int(nz), int(nx), int(nabc), int(nt), float(dt), float(dx), engine.FD_ORDERS[fd_order],
                          bool(free_surface))
    sx, sz = engine._i64(src_x)[:src_n], engine._i64(src_z)[:src_n]
    rx, rz = engine._i64(rcv_x)[:rcv_n], engine._i64(rcv_z)[:rcv_n]
    if sx.size != src_n or rx.size != rcv_n:
        raise ValueError("src_n / rcv_n exceed the position arrays")
    plan = engine.get_plan(geo, sx, sz, rx, rz)

    w = _as_f32(src_v, device, "src_v")
    if w.dim() == 1:
        w = w.unsqueeze(0).expand(src_n, -1)
    if w.shape[-1] != nt:
        raise ValueError(f"src_v has {w.shape[-1]} samples, nt={nt}")
    w = w.contiguous()
    damp_t = _as_f32(damp, device, "damp")
    Nz, Nx = int(nz) + 2 * int(nabc), int(nx) + 2 * int(nabc)
    if tuple(damp_t.shape) != (Nz, Nx):
        raise ValueError(f"damp must have shape {(Nz, Nx)}, got {tuple(damp_t.shape)}")
    for name, t in (("vp", vp), ("rho", rho)):
        if tuple(t.shape) != (int(nz), int(nx)):
            raise ValueError(f"{name} must have shape {(int(nz), int(nx))}, got {tuple(t.shape)}")
    vmax = engine.check_model_inputs(_as_f32(vp, device, "vp"), _as_f32(rho, device, "rho"), w, dt, dx, fd_order)

    wave_grad = torch.is_grad_enabled() and w.requires_grad
    if wave_grad:
        # the adjoint keeps lambda_p on the pressure update region only
        fs = int(nabc) if free_surface else 1
        R = engine.FD_ORDERS[fd_order]
        pz, px = sz + int(nabc), sx + int(nabc)
        if ((pz < max(fs + 1, R)) | (pz > Nz - 1 - R) | (px < R) | (px > Nx - 1 - R)).any():
            raise NotImplementedError("wavelet gradients need every source inside the pressure update region "
                                      f"(no closer than {R} cells to the padded edge, below the free surface)")
    needs_grad_now = torch.is_grad_enabled() and (getattr(vp, "requires_grad", False) or
                                                  getattr(rho, "requires_grad", False) or wave_grad)
    if absorbing == "cpml":
        if needs_grad_now:
            # the CPML adjoint reads every step's imaging fields: no recompute
            if imaging_cache not in ("auto", "all"):
                raise ValueError("CPML gradients keep the imaging fields of every step (imaging_cache='all')")
            imaging_cache = "all"
        plan.set_absorbing("cpml", vmax)
    else:
        plan.set_absorbing(absorbing)
    if autotune is None:
        autotune = os.environ.get("GEOBRAIN_B200_AUTOTUNE", "0") not in ("", "0")
    if autotune and plan.tuned is None:
        vp_a = _as_f32(vp.detach() if torch.is_tensor(vp) else vp, device, "vp")
        rho_a = _as_f32(rho.detach() if torch.is_tensor(rho) else rho, device, "rho")
        plan.autotune(vp_a, rho_a, damp_t, w)

    needs_grad = needs_grad_now
    if needs_grad:
        return engine.differentiable_forward(plan, vp, rho, damp_t, w, device=device,
                                             snapshot_every=int(snapshot_every),
                                             checkpoint_segments=int(checkpoint_segments),
                                             checkpoint_every=int(checkpoint_every),
                                             snapshot_dtype=snapshot_dtype, want_energy=want_energy,
                                             imaging_cache=imaging_cache, imaging_dtype=imaging_dtype,
                                             memory_budget=memory_budget)
    vp_t = _as_f32(vp.detach() if torch.is_tensor(vp) else vp, device, "vp")
    rho_t = _as_f32(rho.detach() if torch.is_tensor(rho) else rho, device, "rho")
    p, vx, vz, en, snaps = engine.run_forward(plan, vp_t, rho_t, damp_t, w, want_energy=want_energy,
                                              snapshot_every=int(snapshot_every))
    return engine.pack_output(plan, p, vx, vz, en, snaps)


# the 3-D kernel lives beside it, under the reference's kernels namespace
from .kernel3d import acoustic_forward_kernel_3d, pad_model_3d  # noqa: E402,F401
