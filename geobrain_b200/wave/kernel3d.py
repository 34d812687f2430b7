"""3-D acoustic forward modelling with the reference's call signature.

``acoustic_forward_kernel_3d`` is a drop-in for
geobrain/physics/wave/kernels/acoustic_3d.py:303-476.  It takes the same
arguments (positions are unpadded grid indices; damp is the padded 3-D
array) and returns the same dict: traces p / vx / vy / vz (src_n, nt, rcv_n)
and energy maps forward_wavefield_{p,vx,vy,vz} (nz, ny, nx).  The CUDA
library (gb3_forward) computes them.  As in the reference, every derivative
is scaled by 1/dz.  When vp or rho requires grad, the traces are
differentiable: the forward keeps every step's imaging fields when they fit
in the device memory (imaging_cache='auto'; no recompute), else checkpoints,
and the backward runs the hand-written adjoint (gb3_backward) in place of
autograd through the reference's time loop.
"""
from __future__ import annotations

import ctypes
import math

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


class _Run3:
    """Validated inputs of one 3-D call, bound to the C ABI."""

    def __init__(self, desc, pos, rpos, damp, w, device):
        self.desc, self.pos, self.rpos, self.damp, self.w, self.device = desc, pos, rpos, damp, w, device
        self.L = _lib.load()

    def check(self, rc):
        if rc == _lib.GB_E_ARG:
            raise ValueError(self.L.gb_last_error().decode())
        _lib.check(rc)

    def forward(self, vp, rho, ckpt=None, K=0, img=None, img_rho=False):
        d, dev = self.desc, self.device
        ws = engine.workspace(int(self.L.gb3_workspace_bytes(ctypes.byref(d))), dev)
        f32 = dict(device=dev, dtype=torch.float32)
        tr = [torch.empty((d.n_shots, d.nt, d.n_rcv), **f32) for _ in range(4)]
        en = [torch.empty((d.nz, d.ny, d.nx), **f32) for _ in range(4)]
        with torch.cuda.device(dev):
            rc = self.L.gb3_forward(ctypes.byref(d), *[p.ctypes.data for p in self.pos],
                                    *[p.ctypes.data for p in self.rpos], vp.data_ptr(), rho.data_ptr(),
                                    self.damp.data_ptr(), self.w.data_ptr(), *[t.data_ptr() for t in tr],
                                    *[e.data_ptr() for e in en], _lib.ptr(ckpt), int(K), _lib.ptr(img),
                                    int(bool(img_rho)), ws.data_ptr(), ws.numel(), engine.stream_handle(dev))
        self.check(rc)
        return tr, en

    def backward(self, vp, rho, res, ckpt, K, want_rho, img=None, img_rho=False, want_wavelet=False):
        d, dev = self.desc, self.device
        K = 0 if img is not None else K
        ws = engine.workspace(int(self.L.gb3_backward_workspace_bytes(ctypes.byref(d), int(K), int(want_rho))), dev)
        gvp = torch.empty((d.nz, d.ny, d.nx), device=dev, dtype=torch.float32)
        grho = torch.empty_like(gvp) if want_rho else None
        gw = torch.empty((d.n_shots, d.nt), device=dev, dtype=torch.float32) if want_wavelet else None
        with torch.cuda.device(dev):
            rc = self.L.gb3_backward(ctypes.byref(d), *[p.ctypes.data for p in self.pos],
                                     *[p.ctypes.data for p in self.rpos], vp.data_ptr(), rho.data_ptr(),
                                     self.damp.data_ptr(), self.w.data_ptr(), *[_lib.ptr(r) for r in res],
                                     _lib.ptr(ckpt), int(K), _lib.ptr(img), int(bool(img_rho)), gvp.data_ptr(),
                                     _lib.ptr(grho), _lib.ptr(gw), ws.data_ptr(), ws.numel(),
                                     engine.stream_handle(dev))
        self.check(rc)
        return gvp, grho, gw


def _imaging_fits(run, nbytes: int) -> bool:
    """Whether nbytes of imaging fields, the adjoint's workspace and a margin
    (2 GiB + 5 %) fit in the device memory available now (counting blocks the
    caching allocator holds unused)."""
    free, _ = torch.cuda.mem_get_info(run.device)
    avail = free + torch.cuda.memory_reserved(run.device) - torch.cuda.memory_allocated(run.device)
    ws = int(run.L.gb3_backward_workspace_bytes(ctypes.byref(run.desc), 0, 1))
    return nbytes + ws + (2 << 30) + avail // 20 <= avail


class _Function3D(torch.autograd.Function):
    """3-D traces as a differentiable function of (vp, rho): every step's
    imaging fields (or checkpoints every K steps) in the forward, the
    hand-written adjoint in the backward (replaces autograd through
    acoustic_3d.py:446-460)."""

    @staticmethod
    def forward(ctx, vp, rho, wavelet, run, K, imaging_cache):
        # the C calls read run.w, the wavelet this graph node differentiates
        run.w = wavelet.detach().contiguous()
        vp32 = vp.detach().to(torch.float32).contiguous()
        rho32 = rho.detach().to(torch.float32).contiguous()
        img_rho = bool(ctx.needs_input_grad[1])
        nimg = int(run.L.gb3_imaging_bytes(ctypes.byref(run.desc), int(img_rho)))
        img = ckpt = None
        if imaging_cache == "auto" and _imaging_fits(run, nimg):
            img = torch.empty(nimg // 4, device=run.device, dtype=torch.float32)
        else:
            ckpt = torch.empty(int(run.L.gb3_checkpoint_bytes(ctypes.byref(run.desc), int(K))) // 4,
                               device=run.device, dtype=torch.float32)
        tr, en = run.forward(vp32, rho32, ckpt, K, img, img_rho)
        ctx.run, ctx.K, ctx.ckpt, ctx.img, ctx.img_rho = run, K, ckpt, img, img_rho
        ctx.save_for_backward(vp32, rho32)
        ctx.mark_non_differentiable(*en)
        return (*tr, *en)

    @staticmethod
    def backward(ctx, gp, gvx, gvy, gvz, *unused):
        vp32, rho32 = ctx.saved_tensors
        need_vp, need_rho, need_w = ctx.needs_input_grad[0], ctx.needs_input_grad[1], ctx.needs_input_grad[2]
        res = [None if t is None else t.to(torch.float32).contiguous() for t in (gp, gvx, gvy, gvz)]
        # img_rho was set from needs_input_grad at the forward, so it covers need_rho
        gvp, grho, gw = ctx.run.backward(vp32, rho32, res, ctx.ckpt, ctx.K, need_rho, ctx.img, ctx.img_rho,
                                         want_wavelet=need_w)
        ctx.ckpt = ctx.img = None
        return (gvp if need_vp else None), (grho if need_rho else None), gw, None, None, None


def acoustic_forward_kernel_3d(nx: int, ny: int, nz: int, dx: float, dy: float, dz: float, nt: int, dt: float,
                               nabc: int, free_surface: bool, src_x: Tensor, src_y: Tensor, src_z: Tensor,
                               src_n: int, src_v: Tensor, rcv_x: Tensor, rcv_y: Tensor, rcv_z: Tensor, rcv_n: int,
                               damp: Tensor, vp: Tensor, rho: Tensor, checkpoint_segments: int = 1,
                               device: torch.device = torch.device("cpu"), dtype: torch.dtype = torch.float32, *,
                               imaging_cache="auto"):
    device = torch.device(device)
    if device.type != "cuda":
        raise ValueError(f"geobrain_b200 runs on CUDA devices only (device={device})")
    if dtype != torch.float32:
        raise TypeError(f"geobrain_b200 computes in float32 (dtype={dtype})")
    if checkpoint_segments < 1:
        raise ValueError(f"checkpoint_segments must be >= 1, got {checkpoint_segments}")
    if imaging_cache not in ("auto", 0):
        raise ValueError(f"imaging_cache must be 'auto' or 0, got {imaging_cache!r}")
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
    for name, t in (("vp", vp), ("rho", rho)):
        if tuple(t.shape) != (nz, ny, nx):
            raise ValueError(f"{name} must have shape {(nz, ny, nx)}, got {tuple(t.shape)}")
    # every derivative is scaled by 1/dz, as in the reference
    engine.check_model_inputs(_as_f32(vp, device, "vp"), _as_f32(rho, device, "rho"), w, dt, dz, 4, ndim=3)
    desc = _lib.Desc3(nz, ny, nx, nabc, nt, src_n, rcv_n, int(bool(free_surface)), float(dt), float(dx), float(dy),
                      float(dz))
    run = _Run3(desc, pos, rpos, damp_t, w, device)
    needs_grad = torch.is_grad_enabled() and (getattr(vp, "requires_grad", False) or
                                              getattr(rho, "requires_grad", False) or w.requires_grad)
    if needs_grad:
        vp_g = vp if torch.is_tensor(vp) else torch.as_tensor(vp)
        rho_g = rho if torch.is_tensor(rho) else torch.as_tensor(rho)
        for name, t in (("vp", vp_g), ("rho", rho_g)):
            if t.device != device:
                raise ValueError(f"{name} is on {t.device}, expected {device}")
        # segments of about sqrt(nt) steps, and never fewer than the caller's checkpoint_segments
        n_seg = max(int(checkpoint_segments), int(math.ceil(math.sqrt(nt))))
        K = max(1, -(-nt // n_seg))
        outs = _Function3D.apply(vp_g, rho_g, w, run, K, imaging_cache)
        tr, en = list(outs[:4]), list(outs[4:])
    else:
        vp_t = _as_f32(vp.detach() if torch.is_tensor(vp) else vp, device, "vp")
        rho_t = _as_f32(rho.detach() if torch.is_tensor(rho) else rho, device, "rho")
        tr, en = run.forward(vp_t, rho_t)
    keys = ("p", "vx", "vy", "vz")
    out = {k: t for k, t in zip(keys, tr)}
    out.update({f"forward_wavefield_{k}": e for k, e in zip(keys, en)})
    return out
