"""Edge cases of the 2-D path through the C ABI against the float64 C
oracle: no receivers, one and two time steps, shot counts that leave a
ragged last shot group, receivers sharing a cell (their adjoint sources add
up), and sources and receivers on the outermost cells the reference can
index.  Tolerances: 1e-5 (forward) and 1e-4 (gradient) relative L2."""
import numpy as np
import pytest
import torch

from conftest import load_case, oracle_kwargs
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def case(nz=30, nx=44, nabc=8, nt=60, n_shots=3, seed=0, free_surface=False):
    from geobrain_b200.wave import RickerWavelet, bc_pml
    rng = np.random.default_rng(seed)
    vp = (1800 + 900 * rng.random((nz, nx))).astype(np.float32)
    rho = (1900 + 400 * rng.random((nz, nx))).astype(np.float32)
    w, _ = RickerWavelet()(f0=25.0, dt=1e-3)
    w = np.pad(w.numpy(), (0, max(0, nt - w.shape[0])))[:nt]
    return dict(nz=nz, nx=nx, nabc=nabc, nt=nt, dt=1e-3, dx=10.0, free_surface=free_surface, vp=vp, rho=rho,
                damp=bc_pml(nx, nz, 10.0, 10.0, nabc, float(vp.max()), free_surface=False).astype(np.float32),
                src_x=rng.integers(0, nx, n_shots).astype(np.int64), src_z=rng.integers(0, nz, n_shots).astype(np.int64),
                src_v=(w[None, :] * (1 + rng.random((n_shots, 1)))).astype(np.float32),
                rcv_x=np.arange(0, nx, 2).astype(np.int64), rcv_z=np.full(nx // 2, 2, np.int64))


def run(c, device, fd_order=4, grad=False, lin=None):
    from geobrain_b200.wave import acoustic_forward_kernel
    vp = torch.tensor(c["vp"], device=device, requires_grad=grad)
    rho = torch.tensor(c["rho"], device=device, requires_grad=grad)
    out = acoustic_forward_kernel(
        nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
        free_surface=c["free_surface"], src_x=c["src_x"], src_z=c["src_z"], src_n=len(c["src_x"]),
        src_v=torch.as_tensor(c["src_v"], device=device), rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
        rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=device), vp=vp, rho=rho, device=device,
        fd_order=fd_order)
    res = {k: v.detach().cpu().numpy() for k, v in out.items()}
    if grad:
        loss = sum((torch.as_tensor(lin[k], device=device, dtype=torch.float32) * out[k]).sum()
                   for k in ("p", "vx", "vz"))
        loss.backward()
        res["grad_vp"], res["grad_rho"] = vp.grad.cpu().numpy(), rho.grad.cpu().numpy()
    torch.cuda.synchronize()
    return res


def lin_weights(c, seed=1):
    rng = np.random.default_rng(seed)
    shape = (len(c["src_x"]), c["nt"], len(c["rcv_x"]))
    return {k: rng.standard_normal(shape) for k in ("p", "vx", "vz")}


def check_forward(c, out, fd_order):
    ref = orc.forward(**oracle_kwargs(c), half=fd_order // 2, dtype=np.float64)
    for k in ("p", "vx", "vz", "forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        assert out[k].shape == ref[k].shape, k
        if ref[k].size and np.abs(ref[k]).max() > 0:
            assert orc.rel_l2(out[k], ref[k]) < 1e-5, (k, orc.rel_l2(out[k], ref[k]))


def check_gradient(c, out, lin, fd_order):
    rvp, rrho, _ = orc.gradient(**oracle_kwargs(c), res_p=lin["p"], res_vx=lin["vx"], res_vz=lin["vz"],
                                half=fd_order // 2, dtype=np.float64)
    assert orc.rel_l2(out["grad_vp"], rvp) < 1e-4, orc.rel_l2(out["grad_vp"], rvp)
    assert orc.rel_l2(out["grad_rho"], rrho) < 1e-4, orc.rel_l2(out["grad_rho"], rrho)


@pytest.mark.parametrize("fd_order", [4, 8])
def test_no_receivers(cuda_device, fd_order):
    c = dict(case(), rcv_x=np.zeros(0, np.int64), rcv_z=np.zeros(0, np.int64))
    out = run(c, cuda_device, fd_order)
    assert out["p"].shape == (3, c["nt"], 0)
    check_forward(c, out, fd_order)


@pytest.mark.parametrize("nt", [1, 2])
@pytest.mark.parametrize("fd_order", [4, 8])
def test_one_and_two_steps(cuda_device, nt, fd_order):
    c = case(nt=nt)
    c["src_v"][:] = 1e3                       # a wavelet that is not zero at the first samples
    lin = lin_weights(c)
    out = run(c, cuda_device, fd_order, grad=True, lin=lin)
    check_forward(c, out, fd_order)
    check_gradient(c, out, lin, fd_order)


@pytest.mark.parametrize("n_shots", [9, 17])
def test_ragged_last_shot_group(cuda_device, n_shots):
    c = case(n_shots=n_shots, nt=50, seed=n_shots)
    lin = lin_weights(c)
    out = run(c, cuda_device, 8, grad=True, lin=lin)
    check_forward(c, out, 8)
    check_gradient(c, out, lin, 8)


@pytest.mark.parametrize("free_surface", [False, True])
def test_shared_receiver_cells_and_border_positions(cuda_device, free_surface):
    """Two receivers on one cell (their adjoint sources add), receivers on
    the last row and column the reference can index, and sources on the
    outermost padded cells."""
    nz, nx, nabc = 30, 44, 8
    c = case(nz=nz, nx=nx, nabc=nabc, nt=70, n_shots=4, seed=5, free_surface=free_surface)
    c["rcv_x"] = np.array([5, 5, -nabc, nx + nabc - 2, 20, 20, 0], np.int64)
    c["rcv_z"] = np.array([3, 3, nz + nabc - 2, -nabc, 0, 0, nz - 1], np.int64)
    c["src_x"] = np.array([-nabc, nx + nabc - 1, 10, 30], np.int64)
    c["src_z"] = np.array([nz + nabc - 1, -nabc, 0, 12], np.int64)
    lin = lin_weights(c, seed=2)
    for fd_order in (4, 8):
        out = run(c, cuda_device, fd_order, grad=True, lin=lin)
        np.testing.assert_array_equal(out["p"][:, :, 0], out["p"][:, :, 1])
        check_forward(c, out, fd_order)
        check_gradient(c, out, lin, fd_order)


def test_unstable_or_non_finite_runs_are_refused(cuda_device):
    """The reference would return Inf / NaN traces; the boundary refuses the
    run before any launch instead, naming the Courant number or the input."""
    c = case()
    with pytest.raises(ValueError, match="Courant"):
        run(dict(c, dt=3e-3), cuda_device, 8)
    bad = dict(c, vp=c["vp"].copy())
    bad["vp"][3, 4] = np.inf
    with pytest.raises(ValueError, match="non-finite"):
        run(bad, cuda_device, 4)
