"""Trace-normalised L2 misfit on the device, fused with its adjoint source.

GeoBrain's FWI example (examples/09_acoustic_fwi.py:290-319) normalises
every trace by its maximum and sums the per-trace L2 norms of the
difference over the traces that are not silent in both.  It does this as
about a dozen torch ops, and autograd then differentiates them.  Here one
CUDA kernel (gb_trace_misfit) computes the loss and, in the same pass, the
exact adjoint source.  ``loss.backward()`` hands that source straight to the
hand-written adjoint as the pressure residual.

    loss = misfit.normalized_trace_l2(out["p"], d_obs)
    loss.backward()                      # vp.grad through the adjoint

One difference: on silent traces and on traces equal to the data after
normalisation, the example's autograd yields NaN (0/0 in the square root's
derivative). Here they yield zero.
"""
from __future__ import annotations

import torch

from .. import _lib
from . import engine


def normalized_trace_l2_with_grad(d_pred: torch.Tensor, d_obs: torch.Tensor):
    """(loss 0-d, dloss/dd_pred, per-trace L (shots, receivers)), float32 on
    d_pred's device; pred and obs are (shots, nt, receivers)."""
    if d_pred.device.type != "cuda":
        raise ValueError(f"geobrain_b200 runs on CUDA devices only (device={d_pred.device})")
    if d_pred.shape != d_obs.shape or d_pred.dim() != 3:
        raise ValueError("d_pred and d_obs must both be (shots, nt, receivers)")
    dev = d_pred.device
    pred = d_pred.detach().to(torch.float32).contiguous()
    obs = d_obs.detach().to(device=dev, dtype=torch.float32).contiguous()
    S, nt, R = pred.shape
    adj = torch.empty_like(pred)
    per = torch.empty((S, R), device=dev, dtype=torch.float32)
    loss = torch.empty((), device=dev, dtype=torch.float32)
    L = _lib.load()
    with torch.cuda.device(dev):
        rc = L.gb_trace_misfit(pred.data_ptr(), obs.data_ptr(), S, nt, R, adj.data_ptr(), per.data_ptr(),
                               loss.data_ptr(), engine.stream_handle(dev))
    _lib.check(rc)
    return loss, adj, per


class _NormalizedL2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, d_pred, d_obs):
        loss, adj, _ = normalized_trace_l2_with_grad(d_pred, d_obs)
        ctx.save_for_backward(adj)
        return loss

    @staticmethod
    def backward(ctx, grad_loss):
        (adj,) = ctx.saved_tensors
        return adj * grad_loss.to(adj.dtype), None


def normalized_trace_l2(d_pred: torch.Tensor, d_obs: torch.Tensor) -> torch.Tensor:
    """The example's misfit as a differentiable 0-d tensor (w.r.t. d_pred)."""
    return _NormalizedL2.apply(d_pred, d_obs)
