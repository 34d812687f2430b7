"""CUDA-graph replay of the gradient's step loops and of the batched engine:
chunks of gb_plan_set_graph_steps steps replayed from one graph (the step
index, and the imaging fields' address, from a device counter) give the
results of one launch per step, bit for bit, with far fewer host launch
calls."""
import numpy as np
import pytest
import torch

from test_batched_gpu import cases, model_dict
from test_forward_gpu import _plan_of, synthetic_case

pytestmark = pytest.mark.gpu


def _unique_receivers(c):
    """Receivers that share a cell add their residuals with shared-memory
    atomics in the adjoint, in an order that varies between runs; keep one
    receiver per cell so that runs can be compared bit for bit."""
    _, keep = np.unique(np.stack([c["rcv_z"], c["rcv_x"]]), axis=1, return_index=True)
    keep = np.sort(keep)
    return dict(c, rcv_x=c["rcv_x"][keep], rcv_z=c["rcv_z"][keep])


def _grad(c, device, **kw):
    from geobrain_b200.wave import acoustic_forward_kernel
    vp = torch.tensor(c["vp"], device=device, requires_grad=True)
    rho = torch.tensor(c["rho"], device=device, requires_grad=kw.pop("want_rho", False))
    out = acoustic_forward_kernel(
        nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
        free_surface=c["free_surface"], src_x=c["src_x"], src_z=c["src_z"], src_n=len(c["src_x"]),
        src_v=torch.as_tensor(c["src_v"], device=device), rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
        rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=device), vp=vp, rho=rho, device=device,
        fd_order=8, **kw)
    lin = np.random.default_rng(5).standard_normal(out["p"].shape).astype(np.float32)
    (out["p"] * torch.as_tensor(lin, device=device)).sum().backward()
    torch.cuda.synchronize()
    return (vp.grad.cpu().numpy(), None if rho.grad is None else rho.grad.cpu().numpy(),
            out["p"].detach().cpu().numpy())


@pytest.mark.parametrize("nt,cache,want_rho", [(100, "all", False), (87, "all", True), (120, "partial", False)])
def test_gradient_graphs_are_bit_identical(cuda_device, nt, cache, want_rho):
    """The forward steps that keep their imaging fields and the adjoint over
    them, replayed in 16-step chunks (an odd cache start, a ragged last chunk,
    the density fields, and a cache over only part of the steps)."""
    c = _unique_receivers(synthetic_case(60, 250, 10, nt, 5, seed=51))
    plan = _plan_of(c, 4)
    ic = "all" if cache == "all" else plan.imaging_bytes(nt // 2 + 7, want_rho, "fp24")
    kw = dict(imaging_cache=ic, imaging_dtype="fp24", checkpoint_every=23, want_rho=want_rho)
    try:
        plan.set_graph_steps(0)
        plan.set_profiling(True)
        base = _grad(c, cuda_device, **kw)
        calls0 = plan.profile()["launch_calls"]
        plan.set_graph_steps(16)
        plan.set_profiling(True)
        outs = [_grad(c, cuda_device, **kw) for _ in range(2)]
        calls1 = plan.profile()["launch_calls"] / 2
    finally:
        plan.set_profiling(False)
        plan.set_graph_steps(16)
    for out in outs:
        for a, b in zip(out, base):
            if b is not None:
                np.testing.assert_array_equal(a, b)
    if cache == "all":
        assert calls1 * 5 < calls0, (calls1, calls0)


def test_batched_graphs_are_bit_identical(cuda_device):
    """Batched forward and adjoint chunks replayed from graphs (models of
    uneven size and step count), against one launch per step."""
    from geobrain_b200.wave import acoustic_forward_batched, acoustic_gradient_batched
    from geobrain_b200.wave.batched import _Prepared
    cs = [_unique_receivers(c) for c in cases()]
    plans = _Prepared([model_dict(c, cuda_device) for c in cs], 8, cuda_device).plans
    obs = [torch.as_tensor(np.random.default_rng(7 + i).standard_normal(
        (len(c["src_x"]), c["nt"], len(c["rcv_x"]))).astype(np.float32), device=cuda_device) for i, c in enumerate(cs)]

    def residual(i, p):
        r = p - obs[i]
        return 0.5 * (r * r).sum(), r

    def run():
        with torch.no_grad():
            fw = acoustic_forward_batched([model_dict(c, cuda_device) for c in cs], fd_order=8, want_energy=False)
        _, g = acoustic_gradient_batched([model_dict(c, cuda_device) for c in cs], residual, fd_order=8)
        return [o["p"].cpu().numpy() for o in fw], [x.cpu().numpy() for x in g]

    try:
        for p in plans:
            p.set_graph_steps(0)
        base = run()
        for p in plans:
            p.set_graph_steps(16)
        out = run()
        out2 = run()
    finally:
        for p in plans:
            p.set_graph_steps(16)
    for o in (out, out2):
        for a, b in zip(o[0] + o[1], base[0] + base[1]):
            np.testing.assert_array_equal(a, b)
