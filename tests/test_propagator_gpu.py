"""The drop-in AcousticPropagator on the GPU against the reference's own
propagator runs (tests/golden/make_golden.py and make_golden_propagator.py
ran geobrain.physics.wave.AcousticPropagator.forward on its CPU path).

  * layered_100x200: the 100 x 200 / 20-cell PML / 1000-step workload
    through the model / survey / propagator API
    (propagators/acoustic.py:150-275): traces and energy maps to 1e-5.
  * propagator_gardner(_fs): AcousticModel(auto_update_rho=True,
    vp_grad=True) (models/acoustic.py:164-195), whose forward() replaces rho
    by Gardner's relation before every propagation; all shots in float32
    (traces, energy maps, the Gardner density), and forward(shot_index=1,
    checkpoint_segments=3) + backward of a loss linear in the traces:
    model.vp.grad against the reference's float64 autograd gradient to 1e-4.
"""
import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-5
GTOL = 1e-4


def _load(name):
    with np.load(f"{GOLDEN}/{name}.npz") as z:
        return {k: z[k] for k in z.files}


def _propagator(c, device, vp_grad, auto_update_rho, rho):
    from geobrain_b200 import wave
    nz, nx, nabc, nt = int(c["nz"]), int(c["nx"]), int(c["nabc"]), int(c["nt"])
    dt, dx, f0 = float(c["dt"]), float(c["dx"]), float(c["f0"])
    grid = wave.GridConfig(nx=nx, nz=nz, dx=dx, dz=dx)
    bnd = wave.BoundaryConfig(type="pml", n_layers=nabc, free_surface=bool(c["free_surface"]))
    model = wave.AcousticModel(grid=grid, boundary=bnd, vp=c["vp"], rho=rho, vp_grad=vp_grad,
                               auto_update_rho=auto_update_rho, device=str(device))
    src = wave.Source(nt=nt, dt=dt, f0=f0)
    for x, z in zip(c["src_x"], c["src_z"]):
        src.add_source(x=int(x), z=int(z), wavelet=c["wavelet"])
    rcv = wave.Receiver(nt=nt, dt=dt)
    rcv.add_receivers(x=c["rcv_x"], z=c["rcv_z"], rcv_type="pr")
    return model, wave.AcousticPropagator(model, wave.Survey(src, rcv), device=str(device))


def test_layered_100x200_propagator_matches_reference(cuda_device):
    c = _load("layered_100x200")
    _, prop = _propagator(c, cuda_device, vp_grad=False, auto_update_rho=False, rho=c["rho"])
    np.testing.assert_allclose(prop.damp.cpu().numpy(), c["damp"], rtol=1e-6, atol=0)
    res = prop.forward()
    for k in ("p", "vx", "vz", "forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        got = getattr(res, k).detach().cpu().numpy()
        assert got.shape == c[f"ref32_{k}"].shape, k
        err = orc.rel_l2(got, c[f"ref32_{k}"])
        assert err < TOL, (k, err)


@pytest.mark.parametrize("name", ["propagator_gardner", "propagator_gardner_fs"])
def test_gardner_propagator_forward_matches_reference(cuda_device, name):
    c = _load(name)
    model, prop = _propagator(c, cuda_device, vp_grad=True, auto_update_rho=True, rho=c["rho0"])
    with torch.no_grad():
        res = prop.forward()
    # Gardner's density, computed in float64 NumPy and cast, as the reference does
    np.testing.assert_allclose(model.rho.detach().cpu().numpy(), c["ref32_rho_gardner"], rtol=1e-6)
    for k in ("p", "vx", "vz", "forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        err = orc.rel_l2(getattr(res, k).cpu().numpy(), c[f"ref32_{k}"])
        assert err < TOL, (k, err)


@pytest.mark.parametrize("name", ["propagator_gardner", "propagator_gardner_fs"])
def test_gardner_propagator_shot_gradient_matches_reference_autograd(cuda_device, name):
    c = _load(name)
    model, prop = _propagator(c, cuda_device, vp_grad=True, auto_update_rho=True, rho=c["rho0"])
    res = prop.forward(shot_index=int(c["shot_index"]), checkpoint_segments=int(c["checkpoint_segments"]))
    assert tuple(res.p.shape) == tuple(c["ref64_shot1_p"].shape)
    assert orc.rel_l2(res.p.detach().cpu().numpy(), c["ref64_shot1_p"]) < TOL
    loss = sum((torch.as_tensor(c[f"lin_{k}"], device=cuda_device, dtype=torch.float32) * getattr(res, k)).sum()
               for k in ("p", "vx", "vz"))
    loss.backward()
    # rho follows vp through Gardner's relation outside autograd: only vp has a gradient
    assert model.rho.grad is None
    err = orc.rel_l2(model.vp.grad.cpu().numpy(), c["ref64_grad_vp"])
    assert err < GTOL, err
