"""Batched propagation of several models of uneven size, step count and
shot count in one launch per step (through the C ABI), against the
single-model path and the CPU oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc
from test_forward_gpu import synthetic_case

pytestmark = pytest.mark.gpu


def model_dict(c, device, requires_grad=False):
    return dict(nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
                free_surface=c["free_surface"], src_x=c["src_x"], src_z=c["src_z"], src_n=len(c["src_x"]),
                src_v=torch.as_tensor(c["src_v"], device=device), rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
                rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=device),
                vp=torch.tensor(c["vp"], device=device, requires_grad=requires_grad),
                rho=torch.tensor(c["rho"], device=device))


CASES = [(60, 130, 10, 70, 3), (45, 250, 8, 110, 5), (90, 121, 12, 90, 2)]


def cases():
    return [synthetic_case(nz, nx, nabc, nt, ns, seed=17 + i) for i, (nz, nx, nabc, nt, ns) in enumerate(CASES)]


def test_batched_forward_matches_single_model_path(cuda_device):
    from geobrain_b200.wave import acoustic_forward_batched, acoustic_forward_kernel
    cs = cases()
    outs = acoustic_forward_batched([model_dict(c, cuda_device) for c in cs], fd_order=8)
    torch.cuda.synchronize()
    for c, o in zip(cs, outs):
        single = acoustic_forward_kernel(**model_dict(c, cuda_device), device=cuda_device, fd_order=8)
        for k in ("p", "vx", "vz"):
            np.testing.assert_array_equal(o[k].cpu().numpy(), single[k].cpu().numpy())
        for k in ("forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
            assert orc.rel_l2(o[k].cpu().numpy(), single[k].cpu().numpy()) < 1e-6
        ref = orc.forward(nz=c["nz"], nx=c["nx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
                          free_surface=False, src_x=c["src_x"], src_z=c["src_z"], src_v=c["src_v"],
                          rcv_x=c["rcv_x"], rcv_z=c["rcv_z"], damp=c["damp"], vp=c["vp"], rho=c["rho"], half=4)
        assert orc.rel_l2(o["p"].cpu().numpy(), ref["p"]) < 1e-5


@pytest.mark.parametrize("imaging_cache,imaging_dtype", [(0, "fp32"), ("auto", "fp32"), ("auto", "fp24"),
                                                         ("auto", "bf16")])
def test_batched_gradient_matches_single_model_path(cuda_device, imaging_cache, imaging_dtype):
    from geobrain_b200.wave import acoustic_forward_batched, acoustic_forward_kernel
    cs = cases()
    rng = np.random.default_rng(0)
    lins = [rng.standard_normal((len(c["src_x"]), c["nt"], len(c["rcv_x"]))).astype(np.float32) for c in cs]
    ms = [model_dict(c, cuda_device, requires_grad=True) for c in cs]
    outs = acoustic_forward_batched(ms, fd_order=8, checkpoint_every=16, imaging_cache=imaging_cache,
                                    imaging_dtype=imaging_dtype)
    loss = sum((torch.as_tensor(l, device=cuda_device) * o["p"]).sum() for l, o in zip(lins, outs))
    loss.backward()
    torch.cuda.synchronize()
    for c, m, l in zip(cs, ms, lins):
        vp = torch.tensor(c["vp"], device=cuda_device, requires_grad=True)
        single = acoustic_forward_kernel(**dict(model_dict(c, cuda_device), vp=vp), device=cuda_device, fd_order=8,
                                         imaging_cache=imaging_cache, imaging_dtype=imaging_dtype)
        (torch.as_tensor(l, device=cuda_device) * single["p"]).sum().backward()
        np.testing.assert_array_equal(m["vp"].grad.cpu().numpy(), vp.grad.cpu().numpy())
    c, l, m = cs[1], lins[1], ms[1]
    rvp, _, _ = orc.gradient(nz=c["nz"], nx=c["nx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
                             free_surface=False, src_x=c["src_x"], src_z=c["src_z"], src_v=c["src_v"],
                             rcv_x=c["rcv_x"], rcv_z=c["rcv_z"], damp=c["damp"], vp=c["vp"], rho=c["rho"],
                             res_p=l.astype(np.float64), half=4)
    assert orc.rel_l2(m["vp"].grad.cpu().numpy(), rvp) < (1e-2 if imaging_dtype == "bf16" else 1e-4)


def test_ensemble_log_likelihood_matches_per_particle_loop(cuda_device):
    """An ensemble of velocity particles through the batched engine
    (sharding.ensemble_forward + sharded_log_likelihood, one process)
    against the reference's per-particle loop of Gaussian log-likelihoods
    (geobrain/core/inverse.py:104-110) over acoustic_forward_kernel."""
    from geobrain_b200.wave import acoustic_forward_kernel, sharding
    c = synthetic_case(40, 90, 10, 80, 2, seed=5)
    template = model_dict(c, cuda_device)
    template.pop("vp")
    rng = np.random.default_rng(1)
    theta = torch.tensor(np.stack([c["vp"] * (1 + 0.02 * rng.standard_normal(c["vp"].shape)) for _ in range(3)])
                         .reshape(3, -1), dtype=torch.float32, device=cuda_device)
    observed = torch.tensor(orc.forward(nz=c["nz"], nx=c["nx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
                                        free_surface=False, src_x=c["src_x"], src_z=c["src_z"], src_v=c["src_v"],
                                        rcv_x=c["rcv_x"], rcv_z=c["rcv_z"], damp=c["damp"], vp=c["vp"],
                                        rho=c["rho"], half=4)["p"], dtype=torch.float32, device=cuda_device)
    fwd = sharding.ensemble_forward(template, (c["nz"], c["nx"]), fd_order=8)
    ll, grad = sharding.sharded_log_likelihood(theta, fwd, observed, noise_std=0.1)
    for i in range(3):
        t = theta[i].clone().reshape(c["nz"], c["nx"]).requires_grad_(True)
        pred = acoustic_forward_kernel(**dict(template, vp=t), device=cuda_device, fd_order=8)["p"]
        r = (pred.reshape(-1) - observed.reshape(-1)) / 0.1
        li = -0.5 * (r * r).sum()
        li.backward()
        assert abs(float(ll[i]) - float(li.detach())) <= 1e-5 * abs(float(li.detach()))
        assert orc.rel_l2(grad[i].reshape(c["nz"], c["nx"]).cpu().numpy(), t.grad.cpu().numpy()) < 1e-5


def test_ensemble_256x512_batched_matches_fp64_oracle(cuda_device):
    """Three particles of the 256 x 512 ensemble workload (8th order, 20-cell
    PML), two shots each, 300 steps, through the batched engine with the
    fp24 imaging cache the benchmark uses: traces of every particle against
    the float64 oracle to 1e-5 and each particle's dL/dvp to 1e-4."""
    from geobrain_b200 import synthetic, wave
    ws = synthetic.ensemble_256x512(n_particles=3, nt=300)
    shots = [1, 6]
    rng = np.random.default_rng(3)
    models, cases, lins = [], [], []
    for w in ws:
        damp = wave.bc_pml(w.nx, w.nz, w.dx, w.dx, w.nabc, float(w.vp.max()), False).astype(np.float32)
        c = dict(nx=w.nx, nz=w.nz, dx=w.dx, nt=w.nt, dt=w.dt, nabc=w.nabc, free_surface=False,
                 src_x=w.src_x[shots], src_z=w.src_z[shots], src_v=np.tile(w.wavelet, (2, 1)).astype(np.float32),
                 rcv_x=w.rcv_x, rcv_z=w.rcv_z, damp=damp, vp=w.vp, rho=w.rho)
        cases.append(c)
        models.append(model_dict(c, cuda_device, requires_grad=True))
        lins.append(rng.standard_normal((2, w.nt, w.rcv_x.size)).astype(np.float32))
    outs = wave.acoustic_forward_batched(models, fd_order=8, want_energy=False, imaging_dtype="fp24")
    loss = sum((torch.as_tensor(l, device=cuda_device) * o["p"]).sum() for l, o in zip(lins, outs))
    loss.backward()
    torch.cuda.synchronize()
    for c, m, o, l in zip(cases, models, outs, lins):
        kw = dict(nz=c["nz"], nx=c["nx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"], free_surface=False,
                  src_x=c["src_x"], src_z=c["src_z"], src_v=c["src_v"], rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
                  damp=c["damp"], vp=c["vp"], rho=c["rho"], half=4)
        ref = orc.forward(**kw, dtype=np.float64)
        assert orc.rel_l2(o["p"].detach().cpu().numpy(), ref["p"]) < 1e-5
        rvp, _, _ = orc.gradient(**kw, res_p=l.astype(np.float64), dtype=np.float64)
        assert orc.rel_l2(m["vp"].grad.cpu().numpy(), rvp) < 1e-4


@pytest.mark.parametrize("budget", [None, "split", "tiny"])
def test_fused_batched_gradient_matches_autograd(cuda_device, budget):
    """acoustic_gradient_batched (forward, residual and adjoint per
    sub-batch, every step's imaging fields kept) gives the autograd batched
    path's gradients bit for bit: with everything in one sub-batch, split
    into sub-batches by a memory budget, and with a budget below one model,
    where each model keeps fp32 checkpoints for the steps that do not fit
    (fp32 restarts reproduce the forward exactly)."""
    from geobrain_b200.wave import acoustic_forward_batched, acoustic_gradient_batched
    from geobrain_b200.wave.batched import _Prepared, full_cache_bytes
    cs = cases()
    rng = np.random.default_rng(2)
    obs = [rng.standard_normal((len(c["src_x"]), c["nt"], len(c["rcv_x"]))).astype(np.float32) for c in cs]
    ms = [model_dict(c, cuda_device, requires_grad=True) for c in cs]
    outs = acoustic_forward_batched(ms, fd_order=8, imaging_dtype="fp24", want_energy=False)
    loss = sum(0.5 * ((o["p"] - torch.as_tensor(d, device=cuda_device)) ** 2).sum() for o, d in zip(outs, obs))
    loss.backward()
    torch.cuda.synchronize()
    mb = None
    if budget is not None:
        prep = _Prepared([model_dict(c, cuda_device) for c in cs], 8, cuda_device)
        sizes = [full_cache_bytes(p, False, "fp24") for p in prep.plans]
        mb = max(sizes) + min(sizes) // 2 if budget == "split" else min(sizes) // 3
    obs_d = [torch.as_tensor(d, device=cuda_device) for d in obs]

    def residual(i, p):
        r = p - obs_d[i]
        return 0.5 * (r * r).sum(), r

    losses, grads = acoustic_gradient_batched([model_dict(c, cuda_device) for c in cs], residual, fd_order=8,
                                              imaging_dtype="fp24", snapshot_dtype="fp32", memory_budget=mb)
    for m, g in zip(ms, grads):
        np.testing.assert_array_equal(g.cpu().numpy(), m["vp"].grad.cpu().numpy())
    assert abs(float(losses.sum()) - float(loss.detach())) <= 1e-5 * abs(float(loss.detach()))

