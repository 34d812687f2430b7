"""Many models in one batch: one kernel launch per time step for all of them.

``acoustic_forward_batched(models)`` takes a list of per-model argument
dicts (the keyword arguments of ``acoustic_forward_kernel``: nx, nz, dx, dz,
nt, dt, nabc, free_surface, src_x, src_z, src_n, src_v, rcv_x, rcv_z, rcv_n,
damp, vp, rho) and returns the list of result dicts.  Models may differ in
grid size, step count, shots and receivers (an SVGD / HMC particle ensemble,
or unrelated models), but share the stencil order and the free-surface
setting.  When any vp / rho requires grad, the traces are differentiable
through the batched hand-written adjoint.

This replaces the serial per-particle loop of GeoBrain's inverse-problem
bridge (geobrain/core/inverse.py:104-110), which calls the propagator once
per particle.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import numpy as np
import torch

from .. import _lib
from . import engine
from .kernel import _as_f32

BATCH_TILE_ROWS = 16


class ModelIO(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in (
        "vp", "rho", "damp", "wavelet", "trace_p", "trace_vx", "trace_vz", "energy_p", "energy_vx", "energy_vz",
        "res_p", "res_vx", "res_vz", "grad_vp", "grad_rho", "store", "workspace")] + [
        ("workspace_bytes", ctypes.c_size_t)]


def _bind():
    return _lib.load()


class _Prepared:
    """Plans, device inputs and sizes of one batch."""

    def __init__(self, models: Sequence[dict], fd_order: int, device):
        if not models:
            raise ValueError("empty batch")
        self.device = device
        self.plans, self.inputs = [], []
        fs0 = bool(models[0].get("free_surface", False))
        for i, m in enumerate(models):
            if bool(m.get("free_surface", False)) != fs0:
                raise ValueError("all models of a batch share the free-surface setting")
            if float(m["dx"]) != float(m.get("dz", m["dx"])):
                raise ValueError(f"model {i}: grid spacing must be equal")
            src_n, rcv_n = int(m["src_n"]), int(m["rcv_n"])
            geo = engine.Geometry(int(m["nz"]), int(m["nx"]), int(m["nabc"]), int(m["nt"]), float(m["dt"]),
                                  float(m["dx"]), engine.FD_ORDERS[fd_order], fs0)
            plan = engine.get_plan(geo, engine._i64(m["src_x"])[:src_n], engine._i64(m["src_z"])[:src_n],
                                   engine._i64(m["rcv_x"])[:rcv_n], engine._i64(m["rcv_z"])[:rcv_n])
            w = _as_f32(m["src_v"], device, "src_v")
            if w.dim() == 1:
                w = w.unsqueeze(0).expand(src_n, -1)
            w = w.contiguous()
            damp = _as_f32(m["damp"], device, "damp")
            try:
                engine.check_model_inputs(_as_f32(m["vp"], device, "vp"), _as_f32(m["rho"], device, "rho"), w,
                                          float(m["dt"]), float(m["dx"]), fd_order)
            except ValueError as e:
                raise ValueError(f"model {i}: {e}") from None
            self.plans.append(plan)
            self.inputs.append((m["vp"], m["rho"], damp, w))
        for plan in self.plans:
            # up to 8 shots per CTA: fewer, longer CTAs measured faster than
            # more, shorter ones even for small models
            plan.set_tiling(BATCH_TILE_ROWS, min(plan.n_shots, 8))
        self.plan_arr = (ctypes.c_void_p * len(self.plans))(*[p.h.value for p in self.plans])


def _forward(prep: _Prepared, vps, rhos, want_energy: bool, stores=None):
    L = _bind()
    dev = prep.device
    n = len(prep.plans)
    ios = (ModelIO * n)()
    keep, outs = [], []
    for i, plan in enumerate(prep.plans):
        g = plan.geo
        S, NR = plan.n_shots, plan.n_rcv
        tr = [torch.empty((S, g.nt, NR), device=dev) for _ in range(3)]
        en = [torch.empty((g.nz, g.nx), device=dev) for _ in range(3)] if want_energy else None
        grad = stores is not None
        ws = engine.workspace(plan.workspace_bytes(False, 0), dev)
        _, _, damp, w = prep.inputs[i]
        io = ios[i]
        io.vp, io.rho, io.damp, io.wavelet = vps[i].data_ptr(), rhos[i].data_ptr(), damp.data_ptr(), w.data_ptr()
        io.trace_p, io.trace_vx, io.trace_vz = [t.data_ptr() for t in tr]
        if en:
            io.energy_p, io.energy_vx, io.energy_vz = [e.data_ptr() for e in en]
        io.store = ctypes.addressof(stores[i]) if grad else None
        io.workspace, io.workspace_bytes = ws.data_ptr(), ws.numel()
        keep.append(ws)
        outs.append((tr, en))
    bws = engine.workspace(L.gb_batch_workspace_bytes(prep.plan_arr, n), dev)
    with torch.cuda.device(dev):
        rc = L.gb_batch_forward(prep.plan_arr, n, ios, bws.data_ptr(), bws.numel(), engine.stream_handle(dev))
    _lib.check(rc)
    return outs


class _BatchFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, prep, opts, *params):
        n = len(prep.plans)
        vps = [p.detach().to(torch.float32).contiguous() for p in params[:n]]
        rhos = [p.detach().to(torch.float32).contiguous() for p in params[n:]]
        dev = prep.device
        K, fmt, with_rho, ifmt = opts["K"], opts["fmt"], opts["with_rho"], opts["imaging_fmt"]
        stores, keep = [], []
        for i, plan in enumerate(prep.plans):
            cached = opts["cached"][i]
            n_ck = -(-(plan.geo.nt - cached) // min(K, plan.geo.nt))
            ck = torch.empty(max(n_ck * plan.checkpoint_bytes(plan.geo.nt, fmt), 256), dtype=torch.uint8, device=dev)
            img = torch.empty(max(plan.imaging_bytes(cached, with_rho, ifmt), 256), dtype=torch.uint8, device=dev)
            stores.append(engine.make_store(ck if n_ck > 0 else None, min(K, plan.geo.nt), fmt,
                                            img if cached > 0 else None, cached, with_rho, ifmt))
            keep.append((ck, img))
        outs = _forward(prep, vps, rhos, opts["want_energy"], stores)
        ctx.prep, ctx.opts, ctx.stores, ctx.keep = prep, opts, stores, keep
        ctx.save_for_backward(*vps, *rhos)
        flat = []
        nondiff = []
        for tr, en in outs:
            if en is None:
                en = [torch.zeros((1,), device=dev) for _ in range(3)]
            flat += tr + en
            nondiff += en
        ctx.mark_non_differentiable(*nondiff)
        return tuple(flat)

    @staticmethod
    def backward(ctx, *grads):
        prep = ctx.prep
        n = len(prep.plans)
        saved = ctx.saved_tensors
        vps, rhos = saved[:n], saved[n:]
        need_vp = any(ctx.needs_input_grad[2:2 + n])
        need_rho = any(ctx.needs_input_grad[2 + n:])
        L = _bind()
        dev = prep.device
        ios = (ModelIO * n)()
        keep, gv, gr = [], [], []
        for i, plan in enumerate(prep.plans):
            g = plan.geo
            res = [None if t is None else t.to(torch.float32).contiguous() for t in grads[6 * i:6 * i + 3]]
            gvp = torch.empty((g.nz, g.nx), device=dev)
            grho = torch.empty((g.nz, g.nx), device=dev) if (need_rho and ctx.stores[i].with_rho) else None
            st = ctx.stores[i]
            seg = max(1, min(st.checkpoint_every, g.nt - st.cached_steps))
            ws = engine.workspace(plan.gradient_workspace_bytes(bool(st.with_rho), seg, ctx.opts["imaging_fmt"]), dev)
            _, _, damp, w = prep.inputs[i]
            io = ios[i]
            io.vp, io.rho, io.damp, io.wavelet = vps[i].data_ptr(), rhos[i].data_ptr(), damp.data_ptr(), w.data_ptr()
            io.res_p, io.res_vx, io.res_vz = [_lib.ptr(r) for r in res]
            io.grad_vp, io.grad_rho = gvp.data_ptr(), _lib.ptr(grho)
            io.store = ctypes.addressof(st)
            io.workspace, io.workspace_bytes = ws.data_ptr(), ws.numel()
            keep.append((ws, res))
            gv.append(gvp)
            gr.append(grho)
        bws = engine.workspace(L.gb_batch_workspace_bytes(prep.plan_arr, n), dev)
        with torch.cuda.device(dev):
            rc = L.gb_batch_backward(prep.plan_arr, n, ios, bws.data_ptr(), bws.numel(), engine.stream_handle(dev))
        _lib.check(rc)
        ctx.keep = None
        out_vp = [g if ctx.needs_input_grad[2 + i] else None for i, g in enumerate(gv)]
        out_rho = [g if ctx.needs_input_grad[2 + n + i] else None for i, g in enumerate(gr)]
        return (None, None, *out_vp, *out_rho)


def _auto_cache_fraction(prep: _Prepared, per_step, K: int, fmt: str, imaging_fmt: str, with_rho: bool,
                         device) -> float:
    """The largest fraction f of every model's steps whose imaging fields the
    forward can keep: the caches, the checkpoints of the other steps, the
    workspaces, the traces and their gradients and a margin (2 GiB + 5 %)
    must fit in the device memory available now."""
    free, _ = torch.cuda.mem_get_info(device)
    avail = free + torch.cuda.memory_reserved(device) - torch.cuda.memory_allocated(device)
    traces = sum(4 * p.n_shots * p.geo.nt * p.n_rcv * 4 for p in prep.plans)   # 3 trace fields + one gradient
    fixed = traces + (2 << 30) + avail // 20 + sum(p.workspace_bytes(False, 0) for p in prep.plans)

    def need(f: float) -> int:
        tot = fixed
        for p, per in zip(prep.plans, per_step):
            nt = p.geo.nt
            c = int(f * nt)
            rest = nt - c
            k = max(1, min(K, nt))
            tot += (c * per + -(-rest // k) * p.checkpoint_bytes(nt, fmt) +
                    p.gradient_workspace_bytes(with_rho, max(1, min(k, rest)), imaging_fmt))
        return tot

    if need(1.0) <= avail:
        return 1.0
    lo, hi = 0.0, 1.0
    if need(0.0) > avail:
        return 0.0
    for _ in range(24):
        mid = 0.5 * (lo + hi)
        if need(mid) <= avail:
            lo = mid
        else:
            hi = mid
    return lo


def acoustic_forward_batched(models: Sequence[dict], *, fd_order: int = 8, device=None, want_energy: bool = True,
                             checkpoint_every: int = 0, snapshot_dtype: str = "fp32",
                             imaging_cache="auto", imaging_dtype: str = "fp32") -> List[dict]:
    """Forward-model every model of `models` together; see the module doc."""
    if fd_order not in engine.FD_ORDERS:
        raise ValueError(f"fd_order must be one of {sorted(engine.FD_ORDERS)}")
    device = torch.device(device if device is not None else models[0]["vp"].device)
    if device.type != "cuda":
        raise ValueError(f"geobrain_b200 runs on CUDA devices only (device={device})")
    for m in models:
        if int(m.get("snapshot_every", 0)) > 0:
            raise ValueError("snapshots are not taken in batched runs; use acoustic_forward_kernel")
    prep = _Prepared(models, fd_order, device)
    vps = [_as_f32(m["vp"], device, "vp") if not torch.is_tensor(m["vp"]) or not m["vp"].requires_grad else m["vp"]
           for m in models]
    rhos = [_as_f32(m["rho"], device, "rho") if not torch.is_tensor(m["rho"]) or not m["rho"].requires_grad
            else m["rho"] for m in models]
    needs_grad = torch.is_grad_enabled() and any(t.requires_grad for t in vps + rhos)
    outs = []
    if not needs_grad:
        res = _forward(prep, [v.detach().float().contiguous() for v in vps],
                       [r.detach().float().contiguous() for r in rhos], want_energy)
        for plan, (tr, en) in zip(prep.plans, res):
            outs.append(engine.pack_output(plan, tr[0], tr[1], tr[2], en, None))
        return outs
    with_rho = any(r.requires_grad for r in rhos)
    K = max(engine.choose_checkpoint_every(p, 1, checkpoint_every, snapshot_dtype, with_rho, imaging_dtype)
            for p in prep.plans)
    # split the imaging-cache budget over the models in proportion to their steps
    if imaging_cache in (0, None, False):
        cached = [0] * len(prep.plans)
    else:
        if imaging_dtype not in _lib.IMAGING_FORMATS:
            raise ValueError(f"imaging_dtype must be one of {sorted(_lib.IMAGING_FORMATS)}")
        per_step = [p.imaging_bytes(1, with_rho, imaging_dtype) for p in prep.plans]
        if imaging_cache == "auto":
            frac = _auto_cache_fraction(prep, per_step, K, snapshot_dtype, imaging_dtype, with_rho, device)
        else:
            total = sum(p.geo.nt * b for p, b in zip(prep.plans, per_step))
            frac = min(1.0, int(imaging_cache) / max(total, 1))
        cached = [int(frac * p.geo.nt) for p in prep.plans]
    opts = dict(K=K, fmt=snapshot_dtype, with_rho=with_rho, want_energy=want_energy, cached=cached,
                imaging_fmt=imaging_dtype)
    flat = _BatchFunction.apply(prep, opts, *vps, *rhos)
    for i, plan in enumerate(prep.plans):
        p, vx, vz, e0, e1, e2 = flat[6 * i:6 * i + 6]
        en = [e0, e1, e2] if want_energy else None
        outs.append(engine.pack_output(plan, p, vx, vz, en, None))
    return outs


def _group_plan_array(plans):
    return (ctypes.c_void_p * len(plans))(*[p.h.value for p in plans])


def _align256(n: int) -> int:
    return (n + 255) // 256 * 256


def full_cache_bytes(plan, with_rho: bool, imaging_dtype: str) -> int:
    """Device bytes one model of a fused batched gradient holds at its peak:
    the imaging fields of every step, the forward and gradient workspaces
    (a one-step segment buffer: nothing is recomputed), the three traces and
    the residual."""
    S, nt, NR = plan.n_shots, plan.geo.nt, plan.n_rcv
    return (plan.imaging_bytes(nt, with_rho, imaging_dtype) + plan.workspace_bytes(False, 0) +
            plan.gradient_workspace_bytes(with_rho, 1, imaging_dtype) + 4 * S * nt * NR * 4)


def plan_sub_batches(sizes: Sequence[int], avail: int) -> List[List[int]]:
    """Split models (in order) into consecutive sub-batches whose summed
    sizes fit in `avail` bytes, as few as fit and as even as they can be: a
    greedy fill first counts the sub-batches, then the smallest per-batch cap
    that still needs no more of them is taken (a greedy fill would leave the
    last sub-batch a few models, too few to fill the GPU).  A model larger
    than `avail` gets a sub-batch of its own (it then keeps checkpoints for
    the steps that do not fit)."""
    def fill(cap: int) -> List[List[int]]:
        groups, cur, tot = [], [], 0
        for i, b in enumerate(sizes):
            if cur and tot + b > cap:
                groups.append(cur)
                cur, tot = [], 0
            cur.append(i)
            tot += b
        if cur:
            groups.append(cur)
        return groups

    groups = fill(avail)
    fitting = [b for b in sizes if b <= avail]
    if len(groups) <= 1 or not fitting:
        return groups
    lo, hi = max(fitting), avail          # fill(hi) needs len(groups) sub-batches
    while lo < hi:
        mid = (lo + hi) // 2
        if len(fill(mid)) <= len(groups):
            hi = mid
        else:
            lo = mid + 1
    return fill(hi)


def acoustic_gradient_batched(models: Sequence[dict], residual, *, fd_order: int = 8, device=None,
                              imaging_dtype: str = "fp24", snapshot_dtype: str = "fp32",
                              memory_budget: Optional[int] = None, with_rho: bool = False):
    """Losses and gradients of many models at once, with the misfit applied
    between the forward and the adjoint (no autograd graph is kept).

    `residual(i, p)` takes model i's pressure traces (n_shots, nt, n_rcv) and
    returns (loss_i, dloss_i/dp) (a 0-d tensor and a tensor like p).  The
    models run in consecutive sub-batches, each as large as the device
    memory allows with the imaging fields of EVERY step kept: a sub-batch
    runs its batched forward (one launch per step for all its models), the
    residuals, and its batched adjoint, then frees its store before the next
    sub-batch starts.  Nothing is recomputed unless one model alone does not
    fit, in which case that model keeps checkpoints (in `snapshot_dtype`)
    for the steps that do not.  memory_budget: the bytes a sub-batch may
    hold (default: the free device memory less 2 GiB and 5 %).  Under
    autograd (acoustic_forward_batched and loss.backward()) every model's
    store must survive until the backward, so
    an ensemble larger than the device memory recomputes its uncached steps;
    this call does not.

    Returns (losses (B,) tensor, [dL/dvp (nz, nx)] per model, and, with
    with_rho, [dL/drho] per model).  The gradients equal those of the
    autograd path, bit for bit, for the same imaging format.  Replaces the
    per-particle forward + backward of InverseProblem.log_likelihood
    (geobrain/core/inverse.py:104-110) for a whole ensemble."""
    if imaging_dtype not in _lib.IMAGING_FORMATS:
        raise ValueError(f"imaging_dtype must be one of {sorted(_lib.IMAGING_FORMATS)}")
    if snapshot_dtype not in _lib.CKPT_FORMATS:
        raise ValueError(f"snapshot_dtype must be one of {sorted(_lib.CKPT_FORMATS)}")
    device = torch.device(device if device is not None else models[0]["vp"].device)
    if device.type != "cuda":
        raise ValueError(f"geobrain_b200 runs on CUDA devices only (device={device})")
    prep = _Prepared(models, fd_order, device)
    n = len(prep.plans)
    vps = [_as_f32(m["vp"].detach() if torch.is_tensor(m["vp"]) else m["vp"], device, "vp") for m in models]
    rhos = [_as_f32(m["rho"].detach() if torch.is_tensor(m["rho"]) else m["rho"], device, "rho") for m in models]
    if memory_budget is not None:
        avail = int(memory_budget)
    else:
        free, _ = torch.cuda.mem_get_info(device)
        avail = free + torch.cuda.memory_reserved(device) - torch.cuda.memory_allocated(device)
        avail -= (2 << 30) + avail // 20
    sizes = [full_cache_bytes(p, with_rho, imaging_dtype) for p in prep.plans]
    losses = torch.zeros(n, dtype=torch.float32, device=device)
    grads_vp, grads_rho = [None] * n, [None] * n
    L = _bind()
    groups = plan_sub_batches(sizes, max(avail, 0))

    def store_layout(group):
        """Per model of a sub-batch: (checkpoint_every, cached steps,
        checkpoint offset and bytes, imaging offset and bytes) in the pool,
        and the sub-batch's total."""
        plans = [prep.plans[i] for i in group]
        if len(group) == 1 and sizes[group[0]] > avail:
            # one model larger than the memory: cache what fits, checkpoint the rest
            p = plans[0]
            K = engine.choose_checkpoint_every(p, 1, 0, snapshot_dtype, with_rho, imaging_dtype)
            cached = engine.choose_cached_steps(p, "auto", with_rho, device, imaging_dtype, K, snapshot_dtype,
                                                memory_budget)
        else:
            K, cached = max(p.geo.nt for p in plans), None
        items, off = [], 0
        for p in plans:
            c = p.geo.nt if cached is None else cached
            n_ck = -(-(p.geo.nt - c) // min(K, p.geo.nt))
            ckb = n_ck * p.checkpoint_bytes(p.geo.nt, snapshot_dtype) if n_ck > 0 else 0
            imb = p.imaging_bytes(c, with_rho, imaging_dtype) if c > 0 else 0
            items.append((K, c, off, ckb, off + _align256(ckb), imb))
            off += _align256(ckb) + _align256(imb)
        return items, off

    # every sub-batch's stores come out of one pool, sized for the largest:
    # allocated once, so the caching allocator is not asked for (and does not
    # fragment on) a new set of blocks per sub-batch of other model sizes
    layouts = [store_layout(g) for g in groups]
    pool = torch.empty(max(max(t for _, t in layouts), 256), dtype=torch.uint8, device=device)
    for group, (items, _) in zip(groups, layouts):
        plans = [prep.plans[i] for i in group]
        arr = _group_plan_array(plans)
        sub = _Sub(prep, group, arr)
        stores = []
        for K, c, ck_off, ckb, im_off, imb in items:
            ck = pool[ck_off:ck_off + ckb] if ckb else None
            img = pool[im_off:im_off + imb] if imb else None
            stores.append(engine.make_store(ck, K, snapshot_dtype, img, c, with_rho, imaging_dtype))
        outs = _forward(sub, [vps[i] for i in group], [rhos[i] for i in group], False, stores)
        res_list = []
        for j, i in enumerate(group):
            p_tr = outs[j][0][0]
            loss_i, res_i = residual(i, p_tr)
            losses[i] = loss_i.detach().to(torch.float32)
            res_list.append(res_i.detach().to(torch.float32).contiguous())
        del outs
        ios = (ModelIO * len(group))()
        wkeep = []
        for j, i in enumerate(group):
            p, st = plans[j], stores[j]
            g = p.geo
            gvp = torch.empty((g.nz, g.nx), device=device)
            grho = torch.empty((g.nz, g.nx), device=device) if with_rho else None
            seg = max(1, min(st.checkpoint_every, g.nt - st.cached_steps))
            ws = engine.workspace(p.gradient_workspace_bytes(with_rho, seg, imaging_dtype), device)
            _, _, damp, w = prep.inputs[i]
            io = ios[j]
            io.vp, io.rho, io.damp, io.wavelet = vps[i].data_ptr(), rhos[i].data_ptr(), damp.data_ptr(), w.data_ptr()
            io.res_p = res_list[j].data_ptr()
            io.grad_vp, io.grad_rho = gvp.data_ptr(), _lib.ptr(grho)
            io.store = ctypes.addressof(st)
            io.workspace, io.workspace_bytes = ws.data_ptr(), ws.numel()
            wkeep.append(ws)
            grads_vp[i], grads_rho[i] = gvp, grho
        bws = engine.workspace(L.gb_batch_workspace_bytes(arr, len(group)), device)
        with torch.cuda.device(device):
            rc = L.gb_batch_backward(arr, len(group), ios, bws.data_ptr(), bws.numel(), engine.stream_handle(device))
        _lib.check(rc)
        del wkeep, res_list, bws
    if with_rho:
        return losses, grads_vp, grads_rho
    return losses, grads_vp


class _Sub:
    """A sub-batch of a _Prepared batch (the plans and inputs of `group`)."""

    def __init__(self, prep: _Prepared, group: Sequence[int], plan_arr):
        self.device = prep.device
        self.plans = [prep.plans[i] for i in group]
        self.inputs = [prep.inputs[i] for i in group]
        self.plan_arr = plan_arr


class AcousticBatch:
    """A fixed list of models, modelled together on every call."""

    def __init__(self, models: Sequence[dict], fd_order: int = 8, device=None):
        self.models = list(models)
        self.fd_order = fd_order
        self.device = device

    def forward(self, vps=None, **kw) -> List[dict]:
        models = self.models
        if vps is not None:
            models = [dict(m, vp=v) for m, v in zip(models, vps)]
        return acoustic_forward_batched(models, fd_order=self.fd_order, device=self.device, **kw)

    __call__ = forward
