"""The CPML absorbing option of the 2-D forward (absorbing='cpml'): the
NumPy oracle's structure against the C oracle, the CUDA path against the
oracle (1e-5 relative L2), and the reason for the option: less reflection
from the grid edges than the damping PML at the same layer width."""
import numpy as np
import pytest
import torch

from conftest import load_case, oracle_kwargs
from oracle import cpml as ocp
from oracle import oracle as orc


@pytest.mark.parametrize("name", ["small_nofs", "small_fs"])
@pytest.mark.parametrize("half", [2, 4])
def test_oracle_without_profiles_is_the_undamped_scheme(name, half):
    """With vanishing profiles the CPML scheme is the reference's leapfrog
    without damping: the oracle reproduces the C oracle run with damp = 0."""
    c = load_case(name)
    kw = oracle_kwargs(c)
    kw.pop("damp")
    a = ocp.forward(**kw, half=half, vmax=1e-30)
    b = orc.forward(**dict(oracle_kwargs(c), damp=np.zeros_like(c["damp"])), half=half, dtype=np.float64)
    for k in ("p", "vx", "vz", "forward_wavefield_p"):
        assert orc.rel_l2(a[k], b[k]) < 1e-12, k


def test_profiles():
    bi, ai, bh, ah = ocp.profiles(60, 10, 10.0, 1e-3, 3000.0, lo=True)
    assert np.all((bi > 0) & (bi <= 1)) and np.allclose(ai, bi - 1)
    assert np.all(ai[10:50] == 0) and np.all(ah[10:49] == 0)       # interior: no absorption
    assert ai[0] < ai[5] < 0 and ai[-1] < ai[-5] < 0               # deeper into the layer: stronger
    bi, ai, _, _ = ocp.profiles(60, 10, 10.0, 1e-3, 3000.0, lo=False)
    assert np.all(ai[:50] == 0)                                    # free surface: no layer on top


def run(c, device, fd_order, **kw):
    from geobrain_b200.wave import acoustic_forward_kernel
    out = acoustic_forward_kernel(
        nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
        free_surface=c["free_surface"], src_x=c["src_x"], src_z=c["src_z"], src_n=len(c["src_x"]),
        src_v=torch.as_tensor(c["src_v"], device=device), rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
        rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=device),
        vp=torch.as_tensor(c["vp"], device=device), rho=torch.as_tensor(c["rho"], device=device), device=device,
        fd_order=fd_order, **kw)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small_nofs", "small_fs"])
@pytest.mark.parametrize("fd_order", [4, 8])
def test_cuda_cpml_matches_oracle(cuda_device, name, fd_order):
    c = load_case(name)
    out = run(c, cuda_device, fd_order, absorbing="cpml")
    kw = oracle_kwargs(c)
    kw.pop("damp")
    ref = ocp.forward(**kw, half=fd_order // 2)
    for k in ("p", "vx", "vz", "forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        assert orc.rel_l2(out[k], ref[k]) < 1e-5, (k, orc.rel_l2(out[k], ref[k]))
    # the damping path on the same plan is untouched
    damped = run(c, cuda_device, fd_order)
    assert orc.rel_l2(damped["p"], orc.forward(**oracle_kwargs(c), half=fd_order // 2, dtype=np.float64)["p"]) < 1e-5


@pytest.mark.gpu
def test_cuda_cpml_graph_replay_and_tilings_are_bit_identical(cuda_device):
    from geobrain_b200.wave import engine
    c = load_case("small_nofs")
    geo = engine.Geometry(c["nz"], c["nx"], c["nabc"], c["nt"], c["dt"], c["dx"], 4, False)
    plan = engine.get_plan(geo, c["src_x"], c["src_z"], c["rcv_x"], c["rcv_z"])
    base = run(c, cuda_device, 8, absorbing="cpml")
    try:
        plan.set_graph_steps(0)
        plan.set_tiling(16, 1)
        other = run(c, cuda_device, 8, absorbing="cpml")
    finally:
        plan.set_graph_steps(16)
        plan.set_tiling(16, 0)
    for k in ("p", "vx", "vz"):
        np.testing.assert_array_equal(other[k], base[k])


@pytest.mark.gpu
def test_cpml_reflects_less_than_the_damping_layers(cuda_device):
    """A homogeneous model with a source near one edge: traces along a line
    close to the edges, against the same model on a grid large enough that
    nothing comes back within nt.  The CPML's edge reflections are a fraction
    of the damping PML's at the same 20-cell width."""
    from geobrain_b200.wave import RickerWavelet, bc_pml
    nz, nx, nabc, nt, dx, dt = 80, 160, 20, 900, 10.0, 1e-3
    w, _ = RickerWavelet()(f0=15.0, dt=dt)
    w = np.pad(w.numpy(), (0, nt))[:nt].astype(np.float32)

    def case(nz_, nx_, off):
        vp = np.full((nz_, nx_), 2500.0, np.float32)
        return dict(nz=nz_, nx=nx_, nabc=nabc, nt=nt, dx=dx, dt=dt, free_surface=False, vp=vp,
                    rho=np.full_like(vp, 2000.0), src_x=np.array([20 + off]), src_z=np.array([40 + off]),
                    src_v=w[None, :], rcv_x=np.arange(0, nx, 4) + off, rcv_z=np.full(nx // 4, 5 + off),
                    damp=bc_pml(nx_, nz_, dx, dx, nabc, 2500.0, False).astype(np.float32))
    small = case(nz, nx, 0)
    big = case(nz + 2 * 400, nx + 2 * 400, 400)          # edges 400 cells away: no return within 0.9 s
    ref = run(big, cuda_device, 8)["p"]
    err_damp = orc.rel_l2(run(small, cuda_device, 8)["p"], ref)
    err_cpml = orc.rel_l2(run(small, cuda_device, 8, absorbing="cpml")["p"], ref)
    assert err_cpml < 0.5 * err_damp, (err_cpml, err_damp)


def _okw(c):
    kw = oracle_kwargs(c)
    kw.pop("damp")
    return kw


@pytest.mark.parametrize("name", ["small_nofs", "small_fs"])
@pytest.mark.parametrize("half", [2, 4])
def test_torch_oracle_is_the_numpy_oracle(name, half):
    """The functional torch restatement (the gradient oracle) computes the
    same traces as the NumPy oracle."""
    c = load_case(name)
    kw = _okw(c)
    vmax = float(np.max(c["vp"]))
    a = ocp.forward(**kw, half=half)
    kt = dict(kw, vp=torch.tensor(c["vp"], dtype=torch.float64), rho=torch.tensor(c["rho"], dtype=torch.float64))
    b = ocp.forward_torch(**kt, half=half, vmax=vmax)
    for k in ("p", "vx", "vz"):
        assert orc.rel_l2(b[k].numpy(), a[k]) < 1e-12, k


def test_torch_oracle_gradient_matches_central_differences():
    """Autograd through the torch oracle against central differences of the
    NumPy oracle along two random directions (float64; vmax held fixed, as
    the layers are built once per plan)."""
    c = load_case("small_fs")
    kw = _okw(c)
    vmax = float(np.max(c["vp"]))
    lin = {k: c[f"lin_{k}"] for k in ("p", "vx", "vz")}
    gvp, grho = ocp.gradient(res_p=lin["p"], res_vx=lin["vx"], res_vz=lin["vz"], half=4, vmax=vmax,
                             **dict(kw, vp=c["vp"], rho=c["rho"]))
    rng = np.random.default_rng(3)

    def loss(vp, rho):
        out = ocp.forward(**dict(kw, vp=vp, rho=rho), half=4, vmax=vmax)
        return sum(float((lin[k] * out[k]).sum()) for k in ("p", "vx", "vz"))

    for g, name in ((gvp, "vp"), (grho, "rho")):
        d = rng.standard_normal(c["vp"].shape)
        base = c[name].astype(np.float64)
        eps = 5e-5 * float(np.abs(base).mean())   # truncation error ~ eps^2: 3e-7 relative here
        args = lambda x: (x, c["rho"].astype(np.float64)) if name == "vp" else (c["vp"].astype(np.float64), x)
        fd = (loss(*args(base + eps * d)) - loss(*args(base - eps * d))) / (2 * eps)
        assert abs(fd - float((g * d).sum())) <= 2e-6 * abs(fd), (name, fd, float((g * d).sum()))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small_nofs", "small_fs"])
@pytest.mark.parametrize("fd_order", [4, 8])
@pytest.mark.parametrize("imaging_dtype", ["fp32", "fp24"])
def test_cuda_cpml_gradient_matches_oracle(cuda_device, name, fd_order, imaging_dtype):
    """dL/dvp and dL/drho of a loss linear in all three traces: the CPML
    adjoint (through the C ABI) against float64 autograd of the torch
    oracle, 1e-4 relative L2."""
    from geobrain_b200.wave import acoustic_forward_kernel
    c = load_case(name)
    S = len(c["src_x"])
    vp = torch.tensor(c["vp"], device=cuda_device, requires_grad=True)
    rho = torch.tensor(c["rho"], device=cuda_device, requires_grad=True)
    out = acoustic_forward_kernel(
        nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
        free_surface=c["free_surface"], src_x=c["src_x"], src_z=c["src_z"], src_n=S,
        src_v=torch.as_tensor(c["src_v"], device=cuda_device), rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
        rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=cuda_device), vp=vp, rho=rho,
        device=cuda_device, fd_order=fd_order, absorbing="cpml", imaging_dtype=imaging_dtype)
    lin = {k: c[f"lin_{k}"] for k in ("p", "vx", "vz")}
    loss = sum((torch.as_tensor(lin[k], device=cuda_device, dtype=torch.float32) * out[k]).sum()
               for k in ("p", "vx", "vz"))
    loss.backward()
    # the traces of a gradient run are the CPML forward's
    ref_tr = ocp.forward(**_okw(c), half=fd_order // 2)
    assert orc.rel_l2(out["p"].detach().cpu().numpy(), ref_tr["p"]) < 1e-5
    rvp, rrho = ocp.gradient(res_p=lin["p"], res_vx=lin["vx"], res_vz=lin["vz"], half=fd_order // 2,
                             vmax=float(np.max(c["vp"])), **dict(_okw(c), vp=c["vp"], rho=c["rho"]))
    assert orc.rel_l2(vp.grad.cpu().numpy(), rvp) < 1e-4, orc.rel_l2(vp.grad.cpu().numpy(), rvp)
    assert orc.rel_l2(rho.grad.cpu().numpy(), rrho) < 1e-4, orc.rel_l2(rho.grad.cpu().numpy(), rrho)


@pytest.mark.gpu
def test_cpml_gradient_needs_the_full_imaging_cache(cuda_device):
    from geobrain_b200.wave import acoustic_forward_kernel
    c = load_case("small_nofs")
    with pytest.raises(ValueError):
        acoustic_forward_kernel(
            nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
            free_surface=False, src_x=c["src_x"], src_z=c["src_z"], src_n=3,
            src_v=torch.as_tensor(c["src_v"], device=cuda_device), rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
            rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=cuda_device),
            vp=torch.tensor(c["vp"], device=cuda_device, requires_grad=True),
            rho=torch.as_tensor(c["rho"], device=cuda_device), device=cuda_device, absorbing="cpml",
            imaging_cache=0)


@pytest.mark.gpu
def test_propagator_cpml_gradient_is_the_kernel_gradient(cuda_device):
    """AcousticPropagator.forward(absorbing='cpml') and loss.backward(), the
    way the FWI example drives the reference, give the kernel's CPML
    gradient; a 3-D model refuses the option instead of ignoring it."""
    from geobrain_b200.wave import (AcousticModel, AcousticPropagator, BoundaryConfig, GridConfig, Receiver,
                                    Source, Survey, acoustic_forward_kernel)
    c = load_case("small_nofs")
    grid = GridConfig(nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"])
    model = AcousticModel(grid, BoundaryConfig(n_layers=c["nabc"]), vp=c["vp"], rho=c["rho"], vp_grad=True,
                          auto_update_rho=False, device=str(cuda_device))
    src = Source(nt=c["nt"], dt=c["dt"], f0=25.0)
    src.add_sources(x=c["src_x"], z=c["src_z"], wavelet=c["src_v"][0])
    rcv = Receiver(nt=c["nt"], dt=c["dt"])
    rcv.add_receivers(x=c["rcv_x"], z=c["rcv_z"], rcv_type="pr")
    prop = AcousticPropagator(model, Survey(src, rcv), device=str(cuda_device))
    lin = torch.as_tensor(c["lin_p"], device=cuda_device, dtype=torch.float32)
    (lin * prop.forward(absorbing="cpml").p).sum().backward()
    g_prop = model.vp.grad.detach().cpu().numpy()

    vp = torch.tensor(c["vp"], device=cuda_device, requires_grad=True)
    out = acoustic_forward_kernel(
        nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
        free_surface=False, src_x=c["src_x"], src_z=c["src_z"], src_n=3,
        src_v=torch.as_tensor(np.tile(c["src_v"][0], (3, 1)), device=cuda_device), rcv_x=c["rcv_x"],
        rcv_z=c["rcv_z"], rcv_n=len(c["rcv_x"]), damp=prop.damp, vp=vp,
        rho=torch.as_tensor(c["rho"], device=cuda_device), device=cuda_device, absorbing="cpml")
    (lin * out["p"]).sum().backward()
    assert orc.rel_l2(g_prop, vp.grad.cpu().numpy()) < 1e-6

    from test_3d import load3
    c3 = load3("small_3d_nofs")
    grid3 = GridConfig(nx=c3["nx"], nz=c3["nz"], dx=c3["dx"], dz=c3["dx"], ny=c3["ny"], dy=c3["dx"])
    m3 = AcousticModel(grid3, BoundaryConfig(n_layers=c3["nabc"]), vp=c3["vp"], rho=c3["rho"], auto_update_rho=False,
                       device=str(cuda_device))
    s3 = Source(nt=c3["nt"], dt=c3["dt"], f0=25.0)
    s3.add_sources(x=c3["src_x"], z=c3["src_z"], y=c3["src_y"], wavelet=c3["src_v"][0])
    r3 = Receiver(nt=c3["nt"], dt=c3["dt"])
    r3.add_receivers(x=c3["rcv_x"], z=c3["rcv_z"], y=c3["rcv_y"], rcv_type="pr")
    with pytest.raises(NotImplementedError):
        AcousticPropagator(m3, Survey(s3, r3), device=str(cuda_device)).forward(absorbing="cpml")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small_nofs", "small_fs"])
def test_cuda_cpml_wavelet_gradient_matches_oracle(cuda_device, name):
    from geobrain_b200.wave import acoustic_forward_kernel
    c = load_case(name)
    w = torch.tensor(c["src_v"], device=cuda_device, requires_grad=True)
    vp = torch.tensor(c["vp"], device=cuda_device, requires_grad=True)
    out = acoustic_forward_kernel(
        nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
        free_surface=c["free_surface"], src_x=c["src_x"], src_z=c["src_z"], src_n=3, src_v=w,
        rcv_x=c["rcv_x"], rcv_z=c["rcv_z"], rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=cuda_device),
        vp=vp, rho=torch.as_tensor(c["rho"], device=cuda_device), device=cuda_device, fd_order=8, absorbing="cpml")
    lin = {k: c[f"lin_{k}"] for k in ("p", "vx", "vz")}
    sum((torch.as_tensor(lin[k], device=cuda_device, dtype=torch.float32) * out[k]).sum() for k in lin).backward()
    rvp, _, rw = ocp.gradient(res_p=lin["p"], res_vx=lin["vx"], res_vz=lin["vz"], half=4, with_wavelet=True,
                              vmax=float(np.max(c["vp"])), **dict(_okw(c), vp=c["vp"], rho=c["rho"]))
    assert orc.rel_l2(w.grad.cpu().numpy(), rw) < 1e-4, orc.rel_l2(w.grad.cpu().numpy(), rw)
    assert orc.rel_l2(vp.grad.cpu().numpy(), rvp) < 1e-4
