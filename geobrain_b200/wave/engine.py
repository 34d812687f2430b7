"""Host-side driver of the C ABI: plans, workspaces, checkpoint storage and
the autograd Function around the hand-written adjoint.

Everything here runs the CUDA library; there is no CPU path.  A call on a
non-CUDA device, in a dtype other than float32, or without the built
library raises.
"""
from __future__ import annotations

import ctypes
import math
import os
from collections import OrderedDict
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from .. import _lib

FD_ORDERS = {4: 2, 8: 4}          # fd_order -> stencil half-width
_PLAN_CACHE: "OrderedDict[tuple, Plan]" = OrderedDict()
_PLAN_CACHE_SIZE = 32


# staggered Taylor coefficients c_k of each order (acoustic_2d.py:211-285 at order 4)
FD_COEFFICIENTS = {4: (9 / 8, 1 / 24), 8: (1225 / 1024, 245 / 3072, 49 / 5120, 5 / 7168)}


def courant_number(vmax: float, dt: float, dx: float, fd_order: int, ndim: int = 2) -> float:
    """Courant number of the staggered leapfrog, vmax dt / dx * sum|c_k| *
    sqrt(ndim); the scheme is stable below 1."""
    return float(vmax) * float(dt) / float(dx) * sum(FD_COEFFICIENTS[fd_order]) * math.sqrt(ndim)


def check_model_inputs(vp: torch.Tensor, rho: torch.Tensor, src_v: torch.Tensor, dt: float, dx: float,
                       fd_order: int, ndim: int = 2) -> float:
    """Host-side checks before a launch (the reference has none: an unstable
    or non-finite run there ends in Inf / NaN traces): vp, rho and the
    wavelets finite, vp and rho positive, and the Courant number below 1.
    One device-to-host read.  Returns vmax."""
    vp, rho, src_v = vp.detach(), rho.detach(), src_v.detach()
    flags = torch.stack([torch.isfinite(vp).all(), torch.isfinite(rho).all(), torch.isfinite(src_v).all(),
                         (vp > 0).all(), (rho > 0).all()]).to(torch.float32)
    vals = torch.cat([flags, vp.max().reshape(1).to(torch.float32)]).tolist()
    for ok, what in zip(vals[:5], ("vp has non-finite values", "rho has non-finite values",
                                   "src_v has non-finite values", "vp must be positive", "rho must be positive")):
        if not ok:
            raise ValueError(what)
    vmax = vals[5]
    cn = courant_number(vmax, dt, dx, fd_order, ndim)
    if cn >= 1.0:
        raise ValueError(f"unstable time step: Courant number {cn:.3f} >= 1 (vmax {vmax:g}, dt {dt:g}, dx {dx:g}, "
                         f"order {fd_order}, {ndim}-D); reduce dt")
    return vmax


def _i64(a) -> np.ndarray:
    if torch.is_tensor(a):
        a = a.detach().cpu().numpy()
    return np.ascontiguousarray(np.atleast_1d(np.asarray(a)).astype(np.int64))


@dataclass(frozen=True)
class Geometry:
    nz: int
    nx: int
    nabc: int
    nt: int
    dt: float
    dx: float
    half: int
    free_surface: bool


class Plan:
    """A gb_plan: validated geometry, receiver binning and workspace sizes."""

    def __init__(self, geo: Geometry, src_x, src_z, rcv_x, rcv_z):
        self.geo = geo
        self.src_x, self.src_z = _i64(src_x), _i64(src_z)
        self.rcv_x, self.rcv_z = _i64(rcv_x), _i64(rcv_z)
        if self.src_x.shape != self.src_z.shape or self.rcv_x.shape != self.rcv_z.shape:
            raise ValueError("position arrays must pair up (x and z of equal length)")
        self.n_shots = int(self.src_x.size)
        self.n_rcv = int(self.rcv_x.size)
        self.desc = _lib.ModelDesc(geo.nz, geo.nx, geo.nabc, geo.nt, self.n_shots, self.n_rcv, geo.half,
                                   int(geo.free_surface), geo.dt, geo.dx)
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        rc = self._lib.gb_plan_create(ctypes.byref(self.desc), self.src_x.ctypes.data, self.src_z.ctypes.data,
                                      self.rcv_x.ctypes.data, self.rcv_z.ctypes.data, ctypes.byref(h))
        if rc != _lib.GB_OK:
            msg = self._lib.gb_last_error().decode()
            raise ValueError(msg) if rc == _lib.GB_E_ARG else _lib.GbError(rc, msg)
        self.h = h
        self.tiling = (0, 0)
        self.group_streams = True
        self.graph_steps = 16                    # the library's default
        self.tuned: Optional[dict] = None       # the autotuner's choice, once it ran

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            self._lib.gb_plan_destroy(h)
            self.h = None

    def set_tiling(self, tile_rows: int = 0, shots_per_cta: int = 0) -> None:
        _lib.check(self._lib.gb_plan_set_tiling(self.h, int(tile_rows), int(shots_per_cta)))
        self.tiling = (tile_rows, shots_per_cta)

    def set_profiling(self, enable: bool) -> None:
        _lib.check(self._lib.gb_plan_set_profiling(self.h, int(enable)))

    def profile(self) -> dict:
        """Milliseconds per phase (forward loop, recompute, adjoint) and kernel
        launches since the last call (needs set_profiling(True))."""
        f, r, a = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        n, calls = ctypes.c_longlong(), ctypes.c_longlong()
        steps = (ctypes.c_longlong * 3)()
        _lib.check(self._lib.gb_plan_launch_calls(self.h, ctypes.byref(calls)))
        _lib.check(self._lib.gb_plan_profile(self.h, ctypes.byref(f), ctypes.byref(r), ctypes.byref(a),
                                             ctypes.byref(n), steps))
        return {"forward_ms": f.value, "recompute_ms": r.value, "adjoint_ms": a.value, "launches": n.value,
                "launch_calls": calls.value, "forward_steps": steps[0], "recompute_steps": steps[1],
                "adjoint_steps": steps[2]}

    def workspace_bytes(self, with_gradient: bool = False, checkpoint_every: int = 0) -> int:
        return int(self._lib.gb_plan_workspace_bytes(self.h, int(with_gradient), int(checkpoint_every)))

    def gradient_workspace_bytes(self, with_rho: bool, segment_steps: int, imaging_fmt: str = "fp32") -> int:
        return int(self._lib.gb_plan_gradient_workspace_bytes(self.h, int(bool(with_rho)), int(segment_steps),
                                                              _lib.IMAGING_FORMATS[imaging_fmt]))

    def checkpoint_bytes(self, checkpoint_every: int, fmt: str) -> int:
        return int(self._lib.gb_plan_checkpoint_bytes(self.h, int(checkpoint_every), _lib.CKPT_FORMATS[fmt]))

    def imaging_bytes(self, cached_steps: int, with_rho: bool = False, fmt: str = "fp32") -> int:
        return int(self._lib.gb_plan_imaging_bytes(self.h, int(cached_steps), int(bool(with_rho)),
                                                   _lib.IMAGING_FORMATS[fmt]))

    def set_group_streams(self, enable: bool) -> None:
        _lib.check(self._lib.gb_plan_set_group_streams(self.h, int(enable)))
        self.group_streams = bool(enable)

    def set_schedule(self, mode: int) -> None:
        """Order of the tile kernels' CTAs (gb_plan_set_schedule): 0 =
        blockIdx order (default), 1 = the slow-path tiles first and the
        forward's last items split in two.  Results are the same either way."""
        _lib.check(self._lib.gb_plan_set_schedule(self.h, int(mode)))

    def set_graph_steps(self, steps: int) -> None:
        """Plain forward as replays of a CUDA graph of `steps` steps (0 = off)."""
        _lib.check(self._lib.gb_plan_set_graph_steps(self.h, int(steps)))
        self.graph_steps = int(steps)

    def autotune(self, vp: torch.Tensor, rho: torch.Tensor, damp: torch.Tensor, src_v: torch.Tensor,
                 steps: int = 16) -> dict:
        """Time `steps` forward steps for every launch configuration
        (gb_plan_autotune) and keep the fastest on this plan."""
        dev = vp.device
        ws = workspace(int(self._lib.gb_plan_autotune_workspace_bytes(self.h)), dev)
        best = ctypes.c_float(0.0)
        with torch.cuda.device(dev):
            rc = self._lib.gb_plan_autotune(self.h, vp.data_ptr(), rho.data_ptr(), damp.data_ptr(), src_v.data_ptr(),
                                            ws.data_ptr(), ws.numel(), int(min(steps, self.geo.nt)),
                                            stream_handle(dev), ctypes.byref(best))
        _lib.check(rc)
        self.tuned = self.config()
        self.tuned["ms_per_step"] = float(best.value)
        return self.tuned

    def config(self) -> dict:
        tz, spc, streams, graph, chunks = (ctypes.c_int() for _ in range(5))
        _lib.check(self._lib.gb_plan_get_config(self.h, ctypes.byref(tz), ctypes.byref(spc), ctypes.byref(streams),
                                                ctypes.byref(graph), ctypes.byref(chunks)))
        return {"tile_rows": tz.value, "shots_per_cta": spc.value, "group_streams": bool(streams.value),
                "graph_steps": graph.value, "stream_chunks": chunks.value,
                "resident_rows": self.resident()["tile_rows"]}

    def set_absorbing(self, mode: str = "damping", vmax: float = 0.0) -> None:
        """'damping' (the reference's damping PML) or 'cpml' (memory-variable
        CPML with a profile for vmax; its gradient needs every step's
        imaging fields in the store)."""
        modes = {"damping": 0, "cpml": 1}
        if mode not in modes:
            raise ValueError(f"absorbing must be one of {sorted(modes)}, got {mode!r}")
        _lib.check(self._lib.gb_plan_set_absorbing(self.h, modes[mode], float(vmax)))

    def set_resident(self, mode, tile_rows: int = 0) -> None:
        """Resident forward: 'auto' (default), False (off), True or 'global'
        (on, edge cells through global memory as (value, tag) words after the
        p and the v updates), 'cluster' (on, edge cells stored into the
        neighbours' shared memory, one cluster of at most 16 CTAs per shot),
        or 'single' (on, one exchange a step: p also updated on the
        neighbours' edge rows and columns; 4th order without a free surface);
        tile_rows 0 (smallest that fits) or one of 4, 8, 12, 16, 24, 32, 36,
        40."""
        m = {"auto": -1, False: 0, True: 1, "global": 1, "cluster": 2, "single": 3}[mode]
        _lib.check(self._lib.gb_plan_set_resident(self.h, m, int(tile_rows)))

    def resident(self) -> dict:
        """The resident forward's tile rows (0: the tile kernel runs), shots
        per launch, and exchange ('global', 'cluster' or 'single')."""
        tz, spl, cl = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(self._lib.gb_plan_get_resident(self.h, ctypes.byref(tz), ctypes.byref(spl), ctypes.byref(cl)))
        return {"tile_rows": tz.value, "shots_per_launch": spl.value,
                "exchange": ("global", "cluster", "single")[cl.value]}

    def set_streaming(self, enable: bool, seg_chunks: int = 0) -> None:
        """Forward steps by the streaming kernel (0 chunks = automatic)."""
        _lib.check(self._lib.gb_plan_set_streaming(self.h, int(bool(enable)), int(seg_chunks)))


def get_plan(geo: Geometry, src_x, src_z, rcv_x, rcv_z) -> Plan:
    sx, sz, rx, rz = _i64(src_x), _i64(src_z), _i64(rcv_x), _i64(rcv_z)
    key = (geo, sx.tobytes(), sz.tobytes(), rx.tobytes(), rz.tobytes())
    plan = _PLAN_CACHE.get(key)
    if plan is None:
        plan = Plan(geo, sx, sz, rx, rz)
        _PLAN_CACHE[key] = plan
        if len(_PLAN_CACHE) > _PLAN_CACHE_SIZE:
            _PLAN_CACHE.popitem(last=False)
    else:
        _PLAN_CACHE.move_to_end(key)
    return plan


def require_cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise ValueError(f"geobrain_b200 runs on CUDA devices only ({name} is on {t.device})")


def workspace(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def stream_handle(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def make_store(checkpoints: Optional[torch.Tensor], checkpoint_every: int, fmt: str,
               imaging: Optional[torch.Tensor], cached_steps: int, with_rho: bool,
               imaging_fmt: str = "fp32") -> "_lib.GradStore":
    return _lib.GradStore(_lib.ptr(checkpoints), int(checkpoint_every), _lib.CKPT_FORMATS[fmt], _lib.ptr(imaging),
                          int(cached_steps), int(bool(with_rho)), _lib.IMAGING_FORMATS[imaging_fmt])


def run_forward(plan: Plan, vp: torch.Tensor, rho: torch.Tensor, damp: torch.Tensor, src_v: torch.Tensor, *,
                want_energy: bool = True, snapshot_every: int = 0, store: Optional["_lib.GradStore"] = None):
    """One gb_forward call.  Returns (p, vx, vz, energies or None, snapshots or None)."""
    g = plan.geo
    dev = vp.device
    S, NR, nt = plan.n_shots, plan.n_rcv, g.nt
    f32 = dict(device=dev, dtype=torch.float32)
    traces = [torch.empty((S, nt, NR), **f32) for _ in range(3)]
    energies = [torch.empty((g.nz, g.nx), **f32) for _ in range(3)] if want_energy else None
    nsnap = (nt + snapshot_every - 1) // snapshot_every if snapshot_every > 0 else 0
    snaps = torch.empty((nsnap, g.nz, g.nx), **f32) if nsnap else None
    ws = workspace(plan.workspace_bytes(False, 0), dev)
    L = plan._lib
    with torch.cuda.device(dev):
        rc = L.gb_forward(plan.h, vp.data_ptr(), rho.data_ptr(), damp.data_ptr(), src_v.data_ptr(),
                          *[t.data_ptr() for t in traces],
                          *([e.data_ptr() for e in energies] if energies else [None, None, None]),
                          int(snapshot_every), _lib.ptr(snaps), ctypes.byref(store) if store is not None else None,
                          ws.data_ptr(), ws.numel(), stream_handle(dev))
    _lib.check(rc)
    return traces[0], traces[1], traces[2], energies, snaps


def pack_output(plan: Plan, p, vx, vz, energies, snaps) -> dict:
    """The dict acoustic_forward_kernel returns (snapshots go to the CPU, as
    in the reference, acoustic_2d.py:484-487)."""
    g = plan.geo
    if energies is None:
        energies = [torch.zeros((g.nz, g.nx), device=p.device, dtype=torch.float32) for _ in range(3)]
    out = {"p": p, "vx": vx, "vz": vz, "forward_wavefield_p": energies[0],
           "forward_wavefield_vx": energies[1], "forward_wavefield_vz": energies[2]}
    if snaps is not None:
        out["snapshots"] = snaps.cpu()
    return out


# ---------------------------------------------------------------------------
# Gradient: checkpointed forward + hand-written adjoint behind autograd
# ---------------------------------------------------------------------------
def choose_checkpoint_every(plan: Plan, checkpoint_segments: int = 1, checkpoint_every: int = 0,
                            fmt: str = "fp32", with_rho: bool = False, imaging_fmt: str = "fp32") -> int:
    """Segment length K: explicit checkpoint_every wins; otherwise the K that
    minimises checkpoint storage + one segment of imaging fields
    (K ~ sqrt(nt * state_bytes / imaging_bytes_per_step)), and never fewer
    segments than the caller's checkpoint_segments asks for."""
    nt = plan.geo.nt
    if checkpoint_every > 0:
        return min(int(checkpoint_every), nt)
    state = plan.checkpoint_bytes(nt, fmt)                             # one stored state
    img_step = plan.imaging_bytes(1, with_rho, imaging_fmt)            # imaging fields of one step
    k = int(max(1, round(math.sqrt(nt * state / max(img_step, 1.0)))))
    k = min(k, max(1, -(-nt // max(1, checkpoint_segments))))
    return max(1, min(k, nt))


def choose_cached_steps(plan: Plan, imaging_cache, with_rho: bool, device, imaging_fmt: str = "fp32",
                        checkpoint_every: int = 1, ckpt_fmt: str = "fp32", memory_budget: Optional[int] = None) -> int:
    """How many of the last time steps keep their imaging fields from the
    forward (those steps skip the recompute).  imaging_cache: a byte budget,
    0, 'all' (every step), or 'auto': the most steps for which the cache, the checkpoints of the
    remaining steps, the workspaces, the trace gradients and a margin (2 GiB
    + 5 %) fit in the device memory available right now, counting blocks the
    caching allocator holds unused (GEOBRAIN_B200_IMAGING_CACHE_BYTES
    overrides it with a byte budget).  memory_budget caps that available
    memory (bytes the whole gradient may hold beyond what is allocated now)."""
    nt = plan.geo.nt
    per = max(plan.imaging_bytes(1, with_rho, imaging_fmt), 1)
    if imaging_cache in (None, 0, False):
        return 0
    if imaging_cache == "all":
        return nt
    if imaging_cache != "auto":
        return int(max(0, min(nt, int(imaging_cache) // per)))
    env = os.environ.get("GEOBRAIN_B200_IMAGING_CACHE_BYTES")
    if env is not None:
        return int(max(0, min(nt, int(env) // per)))
    free, _ = torch.cuda.mem_get_info(device)
    # blocks torch's allocator holds but does not use are free for this too
    avail = free + torch.cuda.memory_reserved(device) - torch.cuda.memory_allocated(device)
    if memory_budget is not None:
        avail = min(avail, int(memory_budget))
    K = max(1, min(int(checkpoint_every), nt))
    one_ck = plan.checkpoint_bytes(nt, ckpt_fmt)                      # one stored state
    fixed = 3 * plan.n_shots * nt * plan.n_rcv * 4 + (2 << 30) + avail // 20

    def need(c: int) -> int:
        rest = nt - c
        seg = max(1, min(K, rest))
        return (c * per + -(-rest // K) * one_ck + plan.gradient_workspace_bytes(with_rho, seg, imaging_fmt) +
                plan.workspace_bytes(0, 0) + fixed)

    if need(nt) <= avail:                # no recompute at all (no segment buffer either)
        return nt
    if need(0) > avail:
        return 0
    lo, hi = 0, nt                       # largest c with need(c) <= avail; every lo kept fits
    while lo < hi:
        mid = (lo + hi + 1) // 2
        if need(mid) <= avail:
            lo = mid
        else:
            hi = mid - 1
    return int(lo)


def run_backward(plan: Plan, vp, rho, damp, src_v, res_p, res_vx, res_vz, store: "_lib.GradStore",
                 want_rho: bool, want_wavelet: bool = False):
    g = plan.geo
    dev = vp.device
    grad_vp = torch.empty((g.nz, g.nx), device=dev, dtype=torch.float32)
    grad_rho = torch.empty((g.nz, g.nx), device=dev, dtype=torch.float32) if want_rho else None
    grad_w = torch.empty((plan.n_shots, g.nt), device=dev, dtype=torch.float32) if want_wavelet else None
    seg = max(1, min(store.checkpoint_every, g.nt - store.cached_steps))    # steps of one recompute segment
    ifmt = {v: k for k, v in _lib.IMAGING_FORMATS.items()}[store.imaging_format]
    ws = workspace(plan.gradient_workspace_bytes(bool(store.with_rho), seg, ifmt), dev)
    with torch.cuda.device(dev):
        rc = plan._lib.gb_backward(plan.h, vp.data_ptr(), rho.data_ptr(), damp.data_ptr(), src_v.data_ptr(),
                                   _lib.ptr(res_p), _lib.ptr(res_vx), _lib.ptr(res_vz), ctypes.byref(store),
                                   grad_vp.data_ptr(), _lib.ptr(grad_rho), _lib.ptr(grad_w), ws.data_ptr(),
                                   ws.numel(), stream_handle(dev))
    _lib.check(rc)
    if want_wavelet:
        return grad_vp, grad_rho, grad_w
    return grad_vp, grad_rho


class AcousticFunction(torch.autograd.Function):
    """Traces (p, vx, vz) as a differentiable function of (vp, rho) and of
    the source wavelets src_v.

    forward: gb_forward keeping checkpoints every K steps (fp32, fp24, or
    bf16 / fp16 with per-snapshot scales) and the imaging fields of the last
    time steps that fit the cache budget; backward: gb_backward (adjoint with
    the imaging condition, fp32 recompute of the uncached segments), in place
    of autograd through ~40 ops per step
    (geobrain/physics/wave/kernels/acoustic_2d.py:448-460)."""

    @staticmethod
    def forward(ctx, vp, rho, plan, damp, src_v, opts):
        dev = vp.device
        src_v = src_v.detach().contiguous()
        vp32 = vp.detach().to(torch.float32).contiguous()
        rho32 = rho.detach().to(torch.float32).contiguous()
        K, fmt, with_rho, cached = opts["checkpoint_every"], opts["fmt"], opts["with_rho"], opts["cached_steps"]
        ifmt = opts["imaging_fmt"]
        n_ck = -(-(plan.geo.nt - cached) // K)
        ckpt = torch.empty(n_ck * plan.checkpoint_bytes(plan.geo.nt, fmt) if n_ck > 0 else 256,
                           dtype=torch.uint8, device=dev)
        img = torch.empty(max(plan.imaging_bytes(cached, with_rho, ifmt), 256), dtype=torch.uint8, device=dev)
        store = make_store(ckpt if n_ck > 0 else None, K, fmt, img if cached > 0 else None, cached, with_rho, ifmt)
        p, vx, vz, en, snaps = run_forward(plan, vp32, rho32, damp, src_v, want_energy=opts["want_energy"],
                                           snapshot_every=opts["snapshot_every"], store=store)
        ctx.plan, ctx.opts = plan, opts
        ctx.store_keep = (ckpt, img)
        ctx.store = store
        ctx.save_for_backward(vp32, rho32, damp, src_v)
        if en is None:
            en = [torch.zeros((plan.geo.nz, plan.geo.nx), device=dev) for _ in range(3)]
        snaps = snaps if snaps is not None else torch.empty(0, device=dev)
        ctx.mark_non_differentiable(*en, snaps)
        return p, vx, vz, en[0], en[1], en[2], snaps

    @staticmethod
    def backward(ctx, gp, gvx, gvz, *unused):
        vp32, rho32, damp, src_v = ctx.saved_tensors
        need_vp, need_rho, need_w = ctx.needs_input_grad[0], ctx.needs_input_grad[1], ctx.needs_input_grad[4]
        if not (need_vp or need_rho or need_w):
            return None, None, None, None, None, None
        res = [None if t is None else t.to(torch.float32).contiguous() for t in (gp, gvx, gvz)]
        if all(r is None for r in res):
            z = torch.zeros_like(vp32)
            return ((z if need_vp else None), (z.clone() if need_rho else None), None, None,
                    (torch.zeros_like(src_v) if need_w else None), None)
        out = run_backward(ctx.plan, vp32, rho32, damp, src_v, *res, ctx.store,
                           need_rho and bool(ctx.store.with_rho), want_wavelet=need_w)
        gvp, grho = out[0], out[1]
        ctx.store_keep = None
        return (gvp if need_vp else None), (grho if need_rho else None), None, None, (out[2] if need_w else None), None


def differentiable_forward(plan: Plan, vp, rho, damp, src_v, *, device, snapshot_every: int = 0,
                           checkpoint_segments: int = 1, checkpoint_every: int = 0, snapshot_dtype: str = "fp32",
                           want_energy: bool = True, imaging_cache="auto", imaging_dtype: str = "fp32",
                           memory_budget: Optional[int] = None) -> dict:
    if snapshot_dtype not in _lib.CKPT_FORMATS:
        raise ValueError(f"snapshot_dtype must be one of {sorted(_lib.CKPT_FORMATS)}")
    if imaging_dtype not in _lib.IMAGING_FORMATS:
        raise ValueError(f"imaging_dtype must be one of {sorted(_lib.IMAGING_FORMATS)}")
    need_rho = bool(getattr(rho, "requires_grad", False))
    vp_t = vp if torch.is_tensor(vp) else torch.as_tensor(vp)
    rho_t = rho if torch.is_tensor(rho) else torch.as_tensor(rho)
    for name, t in (("vp", vp_t), ("rho", rho_t)):
        if t.device != device:
            raise ValueError(f"{name} is on {t.device}, expected {device}")
    K = choose_checkpoint_every(plan, checkpoint_segments, checkpoint_every, snapshot_dtype, need_rho, imaging_dtype)
    cached = choose_cached_steps(plan, imaging_cache, need_rho, device, imaging_dtype, K, snapshot_dtype,
                                 memory_budget)
    opts = dict(checkpoint_every=K, fmt=snapshot_dtype, want_energy=want_energy, snapshot_every=snapshot_every,
                with_rho=need_rho, cached_steps=cached, imaging_fmt=imaging_dtype)
    p, vx, vz, e0, e1, e2, snaps = AcousticFunction.apply(vp_t, rho_t, plan, damp, src_v, opts)
    out = {"p": p, "vx": vx, "vz": vz, "forward_wavefield_p": e0, "forward_wavefield_vx": e1,
           "forward_wavefield_vz": e2}
    if snapshot_every > 0:
        out["snapshots"] = snaps.detach().cpu()
    return out
