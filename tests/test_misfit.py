"""The trace-normalised L2 misfit of GeoBrain's FWI example
(examples/09_acoustic_fwi.py:290-319): the float64 oracle against torch
autograd of the example's own expression (CPU), then the CUDA kernel behind
wave.misfit against the oracle (GPU, through the C ABI)."""
import numpy as np
import pytest
import torch

from oracle import misfit as om
from oracle import oracle as orc


def reference_expression(d_pred, d_obs):
    """examples/09_acoustic_fwi.py:290-319, restated in torch."""
    def normalize_traces(data):
        max_vals = torch.max(torch.abs(data), dim=-2, keepdim=True).values
        max_vals = max_vals.clamp(min=1e-30)
        return data / max_vals
    residual = normalize_traces(d_obs) - normalize_traces(d_pred)
    per_trace_l2 = torch.sqrt(torch.sum(residual ** 2, dim=-2))
    trace_energy_obs = torch.sum(torch.abs(d_obs), dim=-2)
    trace_energy_syn = torch.sum(torch.abs(d_pred), dim=-2)
    active_mask = ~((trace_energy_obs == 0) & (trace_energy_syn == 0))
    return torch.sum(per_trace_l2[active_mask])


def edge_case_traces(S=3, nt=57, R=11, seed=0):
    """Random traces plus every edge case of the expression: a silent trace
    in both, a silent prediction with live data, a silent observation, ties
    in the maximum, a trace below the clamp, and a prediction equal to the
    data up to scale (L = 0)."""
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((S, nt, R))
    o = rng.standard_normal((S, nt, R))
    d[0, :, 0] = 0.0
    o[0, :, 0] = 0.0                      # inactive
    d[0, :, 1] = 0.0                      # silent prediction, live data
    o[1, :, 2] = 0.0                      # silent data, live prediction
    d[1, :, 3] = 0.0
    d[1, 5, 3], d[1, 9, 3] = -2.0, 2.0    # tie in |d|: the first index takes the max's gradient
    d[2, :, 4] *= 1e-32                   # below the clamp
    o[2, :, 5] = d[2, :, 5]               # L = 0
    return d, o


def test_oracle_matches_autograd_of_the_reference_expression():
    d, o = edge_case_traces()
    dt = torch.tensor(d, requires_grad=True)
    loss = reference_expression(dt, torch.tensor(o))
    loss.backward()
    ref = dt.grad.numpy()
    got_loss, got, per = om.normalized_trace_l2(d, o)
    assert abs(got_loss - float(loss)) <= 1e-12 * abs(float(loss))
    # autograd's 0/0 in the square root's derivative: at L = 0, and on the
    # masked-out silent trace (its zero upstream gradient still passes
    # through sqrt(0)); the oracle (and the kernel) give zeros there
    nan_traces = np.isnan(ref).any(axis=1)
    assert nan_traces[2, 5] and nan_traces[0, 0] and nan_traces.sum() == 2
    assert not got[2, :, 5].any() and not got[0, :, 0].any()
    keep = ~nan_traces
    np.testing.assert_allclose(got.transpose(0, 2, 1)[keep], ref.transpose(0, 2, 1)[keep], rtol=1e-10,
                               atol=1e-12 * np.abs(ref[~np.isnan(ref)]).max())
    assert per[0, 0] == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(3, 57, 11), (2, 3000, 1200), (1, 1, 1)])
def test_cuda_misfit_matches_oracle(cuda_device, shape):
    from geobrain_b200.wave import misfit
    S, nt, R = shape
    d, o = edge_case_traces(S, nt, R) if shape == (3, 57, 11) else (
        np.random.default_rng(1).standard_normal(shape), np.random.default_rng(2).standard_normal(shape))
    d32, o32 = d.astype(np.float32), o.astype(np.float32)
    loss, adj, per = misfit.normalized_trace_l2_with_grad(torch.tensor(d32, device=cuda_device),
                                                          torch.tensor(o32, device=cuda_device))
    ref_loss, ref_adj, ref_per = om.normalized_trace_l2(d32, o32)
    assert abs(float(loss) - ref_loss) <= 1e-5 * abs(ref_loss)
    assert orc.rel_l2(adj.cpu().numpy(), ref_adj) < 1e-5
    assert orc.rel_l2(per.cpu().numpy(), ref_per) < 1e-5


@pytest.mark.gpu
def test_cuda_misfit_autograd_feeds_the_adjoint(cuda_device):
    """loss.backward() through the misfit hands its adjoint source to the
    hand-written adjoint: the vp gradient equals the oracle's gradient with
    the oracle misfit's residual."""
    from conftest import load_case, oracle_kwargs
    from geobrain_b200.wave import acoustic_forward_kernel, misfit
    c = load_case("small_nofs")
    vp = torch.tensor(c["vp"], device=cuda_device, requires_grad=True)
    out = acoustic_forward_kernel(
        nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
        free_surface=False, src_x=c["src_x"], src_z=c["src_z"], src_n=3,
        src_v=torch.as_tensor(c["src_v"], device=cuda_device), rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
        rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=cuda_device), vp=vp,
        rho=torch.as_tensor(c["rho"], device=cuda_device), device=cuda_device, fd_order=8)
    d_obs = torch.tensor(c["ref32_p"] * 0.7 + 1e-7, device=cuda_device)
    loss = misfit.normalized_trace_l2(out["p"], d_obs)
    loss.backward()
    pred = out["p"].detach().cpu().numpy()
    ref_loss, ref_adj, _ = om.normalized_trace_l2(pred, d_obs.cpu().numpy())
    assert abs(float(loss.detach()) - ref_loss) <= 1e-5 * ref_loss
    rvp, _, _ = orc.gradient(**oracle_kwargs(c), res_p=ref_adj, half=4, dtype=np.float64)
    assert orc.rel_l2(vp.grad.cpu().numpy(), rvp) < 1e-4
