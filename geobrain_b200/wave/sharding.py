"""Shot and model sharding across GPUs: one process per GPU, independent
work per rank, one all-reduce at the end.

The path has no exchange between shots or between models.  The only
collective is the sum of each rank's partial results: the (nz, nx) gradient
and the misfit of an FWI gradient over shots, or the per-particle
log-likelihoods and their gradients of an ensemble.  Each sum is packed into
one buffer and reduced with one ``all_reduce`` (NCCL over NVLink on GPUs,
gloo on CPU).  There is no domain decomposition.

This replaces two serial loops of the reference:
- the per-particle loop of ``InverseProblem.log_likelihood``
  (geobrain/core/inverse.py:104-110), see ``sharded_log_likelihood``;
- the single-process shot loop behind ``AcousticPropagator.forward``
  (geobrain/physics/wave/propagators/acoustic.py:205-273), see
  ``sharded_shot_gradient``.

Both take the rank-local computation as a function, so the same host logic
drives the CUDA engine (``fwi_local_fn``, ``acoustic_forward_batched``) and
any other forward model.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import torch
import torch.distributed as dist


def _world(group) -> Tuple[int, int]:
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(group), dist.get_rank(group)
    return 1, 0


def partition(weights: Sequence[float], world: int, rank: int) -> List[int]:
    """Indices of the items that rank `rank` of `world` takes.

    Longest-processing-time assignment: items in decreasing weight (ties by
    index) go to the least-loaded rank (ties by rank).  The result is
    deterministic, so every rank computes the same split without
    communicating.  Each rank's indices come back in increasing order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    w = [float(x) for x in weights]
    if any(x < 0 for x in w):
        raise ValueError("weights must be non-negative")
    load = [0.0] * world
    owner = [0] * len(w)
    for i in sorted(range(len(w)), key=lambda i: (-w[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        owner[i] = r
        load[r] += w[i]
    return [i for i in range(len(w)) if owner[i] == rank]


def allreduce_packed(tensors: Sequence[torch.Tensor], group=None) -> List[torch.Tensor]:
    """Sum each tensor over the ranks of `group` with ONE all_reduce: the
    tensors are flattened into one buffer (of the first tensor's dtype and
    device), reduced, and split back into new tensors of the input shapes."""
    world, _ = _world(group)
    if world == 1:
        return [t.detach().clone() for t in tensors]
    dtype, device = tensors[0].dtype, tensors[0].device
    buf = torch.cat([t.detach().reshape(-1).to(dtype=dtype, device=device) for t in tensors])
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    out, o = [], 0
    for t in tensors:
        n = t.numel()
        out.append(buf[o:o + n].reshape(t.shape).to(t.dtype))
        o += n
    return out


def sharded_shot_gradient(n_shots: int, local_fn: Callable[[List[int]], Tuple[torch.Tensor, torch.Tensor]],
                          group=None, weights: Optional[Sequence[float]] = None):
    """Misfit and gradient of a multi-shot objective, shots split over ranks.

    local_fn(shots) returns (loss, grad) for the listed shot indices: a
    0-d loss tensor and the model-shaped gradient.  An empty list must give
    zeros, for a rank that gets no shot.  Every rank returns the totals over
    all shots."""
    world, rank = _world(group)
    mine = partition(weights if weights is not None else [1.0] * n_shots, world, rank)
    loss, grad = local_fn(mine)
    loss_sum, grad_sum = allreduce_packed([grad, loss.reshape(1)], group)[::-1]
    return loss_sum.reshape(()), grad_sum


def fwi_local_fn(kernel_kwargs: dict, vp: torch.Tensor, rho: torch.Tensor, d_obs: torch.Tensor,
                 misfit: Optional[Callable[[torch.Tensor, torch.Tensor], torch.Tensor]] = None, **kw):
    """The rank-local part of an FWI gradient on the CUDA engine.

    kernel_kwargs are the arguments of acoustic_forward_kernel except
    vp / rho (src_x, src_z, src_v over ALL shots); d_obs is (n_shots, nt,
    n_rcv).  The returned function models the listed shots, applies
    `misfit(pred, obs)` (default ½‖pred − obs‖²) and returns the loss and
    dL/dvp."""
    from .kernel import acoustic_forward_kernel

    if misfit is None:
        def misfit(pred, obs):
            r = pred - obs
            return 0.5 * (r * r).sum()

    def run(shots: List[int]):
        if not shots:
            return torch.zeros((), device=vp.device), torch.zeros_like(vp)
        idx = torch.as_tensor(shots, dtype=torch.long)
        args = dict(kernel_kwargs)
        sel = lambda a: (a[idx.to(a.device)] if torch.is_tensor(a) else torch.as_tensor(a)[idx]).contiguous()
        args["src_x"], args["src_z"] = sel(args["src_x"]), sel(args["src_z"])
        w = args["src_v"]
        args["src_v"] = sel(w) if torch.as_tensor(w).dim() == 2 else w
        args["src_n"] = len(shots)
        v = vp.detach().requires_grad_(True)
        out = acoustic_forward_kernel(vp=v, rho=rho, **args, **kw)
        loss = misfit(out["p"], d_obs[idx.to(d_obs.device)])
        loss.backward()
        return loss.detach(), v.grad

    return run


def ensemble_forward(template: dict, model_shape, **kw) -> Callable[[torch.Tensor], torch.Tensor]:
    """forward_batch for sharded_log_likelihood on the CUDA engine: each
    particle, reshaped to `model_shape` (nz, nx), is the vp of one model of
    `template` (the acoustic_forward_kernel arguments shared by all
    particles), and the batch runs through acoustic_forward_batched (one
    launch per time step for all of them, differentiable).  Returns the
    pressure traces, (b, n_shots, nt, n_rcv)."""
    from .batched import acoustic_forward_batched

    def forward_batch(theta_local: torch.Tensor) -> torch.Tensor:
        models = [dict(template, vp=t.reshape(model_shape).float()) for t in theta_local]
        outs = acoustic_forward_batched(models, **kw)
        return torch.stack([o["p"] for o in outs])

    return forward_batch


def ensemble_value_and_grad(template: dict, model_shape, observed: torch.Tensor, noise_std: float = 1.0,
                            **kw) -> Callable[[torch.Tensor], Tuple[torch.Tensor, torch.Tensor]]:
    """value_and_grad for sharded_log_likelihood on the CUDA engine: the
    Gaussian log-likelihoods ll_i = -½ ‖(F(θ_i) − D) / σ‖² of a batch of
    velocity particles and d ll_i / d θ_i, by acoustic_gradient_batched (the
    misfit is applied between the batched forward and the batched adjoint,
    in sub-batches that keep every step's imaging fields, so nothing is
    recomputed).  Same values as autograd through ensemble_forward."""
    from .batched import acoustic_gradient_batched

    def value_and_grad(theta_local: torch.Tensor):
        models = [dict(template, vp=t.detach().reshape(model_shape).float()) for t in theta_local]
        obs = observed.reshape(-1)
        inv_var = 1.0 / (noise_std * noise_std)

        def residual(i, p):
            r = p.reshape(-1) - obs.to(p.dtype)
            return 0.5 * inv_var * (r * r).sum(), (inv_var * r).reshape(p.shape)

        losses, grads = acoustic_gradient_batched(models, residual, **kw)
        return -losses.to(theta_local.dtype), -torch.stack([g.reshape(-1) for g in grads]).reshape(
            theta_local.shape).to(theta_local.dtype)

    return value_and_grad


def sharded_log_likelihood(theta: torch.Tensor, forward_batch: Optional[Callable[[torch.Tensor], torch.Tensor]],
                           observed: torch.Tensor, noise_std: float = 1.0, group=None,
                           weights: Optional[Sequence[float]] = None, with_grad: bool = True,
                           value_and_grad: Optional[Callable] = None):
    """Gaussian log-likelihoods (and their gradients) of a batch of
    particles, particles split over ranks (InverseProblem.log_likelihood,
    geobrain/core/inverse.py:81-110, without its per-particle loop).

    forward_batch(theta_local) maps (b, ...) particles to (b, ...)
    predictions in one call (acoustic_forward_batched for an ensemble of
    velocity models).  ll_i = -½ ‖(F(θ_i) − D) / σ‖².  Returns (ll, grad):
    ll of shape (B,), grad = d ll_i / d θ_i of theta's shape (None without
    with_grad), the same on every rank.  With value_and_grad (for instance
    ensemble_value_and_grad), value_and_grad(theta_local) gives the local
    (ll, grad) directly and forward_batch is used only without with_grad."""
    world, rank = _world(group)
    B = theta.shape[0]
    mine = partition(weights if weights is not None else [1.0] * B, world, rank)
    ll_full = torch.zeros(B, dtype=theta.dtype, device=theta.device)
    grad_full = torch.zeros_like(theta) if with_grad else None
    if mine and with_grad and value_and_grad is not None:
        idx = torch.as_tensor(mine, dtype=torch.long, device=theta.device)
        ll, g = value_and_grad(theta.detach()[idx])
        grad_full[idx] = g.to(grad_full.dtype)
        ll_full[idx] = ll.detach().to(ll_full.dtype)
    elif mine:
        idx = torch.as_tensor(mine, dtype=torch.long, device=theta.device)
        th = theta.detach()[idx].clone().requires_grad_(with_grad)
        with torch.set_grad_enabled(with_grad):
            pred = forward_batch(th)
            res = (pred.reshape(len(mine), -1) - observed.reshape(1, -1).to(pred.dtype)) / noise_std
            ll = -0.5 * (res * res).sum(dim=1)
        if with_grad:
            (g,) = torch.autograd.grad(ll.sum(), th)
            grad_full[idx] = g.to(grad_full.dtype)
        ll_full[idx] = ll.detach().to(ll_full.dtype)
    if with_grad:
        ll_full, grad_full = allreduce_packed([ll_full, grad_full], group)
    else:
        (ll_full,) = allreduce_packed([ll_full], group)
    return ll_full, grad_full
