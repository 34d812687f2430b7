"""CPU oracle of the trace-normalised L2 misfit of GeoBrain's FWI example
and of its exact gradient (the adjoint source).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA
misfit kernel.  The product package never imports it.

Restates examples/09_acoustic_fwi.py:290-319 in float64 NumPy.  For traces
d (shots, nt, receivers) and observations o of the same shape:

    m_d = max(max_t |d_t|, 1e-30),  m_o likewise              (:295-299)
    r_t = o_t / m_o - d_t / m_d                                (:310-312)
    L_j = sqrt(sum_t r_t^2)   per trace j = (shot, receiver)    (:313)
    active_j = not (sum_t |o_t| == 0 and sum_t |d_t| == 0)      (:316-318)
    loss = sum over active traces of L_j                        (:320)

Gradient w.r.t. d, as autograd through that expression gives it.  With
g_t = -r_t / L_j and t* the first time index of the largest |d_t|:

    dloss/dd_t = g_t / m_d - [t == t*] sign(d_t*) (sum_u g_u d_u) / m_d^2

The second term is the max's gradient; it is absent when max|d| < 1e-30
(the clamp passes no gradient).  Inactive traces and traces with L_j = 0
(prediction equal to the data after normalisation) get zero.  Autograd
through the example's expression gives NaN on both (0/0 in the square
root's derivative, which the mask does not stop), and one NaN would spoil
the whole model gradient.
"""
from __future__ import annotations

import numpy as np

CLAMP = 1e-30


def normalized_trace_l2(pred: np.ndarray, obs: np.ndarray):
    """(loss, dloss/dpred, per-trace L (shots, receivers)) in float64."""
    d = np.asarray(pred, dtype=np.float64)
    o = np.asarray(obs, dtype=np.float64)
    if d.shape != o.shape or d.ndim != 3:
        raise ValueError("pred and obs must both be (shots, nt, receivers)")
    ad = np.abs(d)
    raw_max = ad.max(axis=1)                                     # (S, R)
    t_star = ad.argmax(axis=1)                                   # first index of the maximum
    m_d = np.maximum(raw_max, CLAMP)
    m_o = np.maximum(np.abs(o).max(axis=1), CLAMP)
    r = o / m_o[:, None, :] - d / m_d[:, None, :]
    L = np.sqrt((r * r).sum(axis=1))
    active = ~((np.abs(o).sum(axis=1) == 0) & (ad.sum(axis=1) == 0))
    loss = float(L[active].sum())

    ok = active & (L > 0)
    Ls = np.where(ok, L, 1.0)
    g = np.where(ok[:, None, :], -r / Ls[:, None, :], 0.0)      # dloss/dn_t
    grad = g / m_d[:, None, :]
    s_gd = (g * d).sum(axis=1)                                   # sum_u g_u d_u
    S, _, R = d.shape
    si, ri = np.meshgrid(np.arange(S), np.arange(R), indexing="ij")
    d_star = d[si, t_star, ri]
    corr = np.where(raw_max >= CLAMP, np.sign(d_star) * s_gd / (m_d * m_d), 0.0)
    grad[si, t_star, ri] -= corr
    return loss, grad, np.where(active, L, 0.0)
