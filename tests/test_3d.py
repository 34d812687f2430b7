"""3-D acoustic path (geobrain/physics/wave/kernels/acoustic_3d.py): the
NumPy oracle against the reference's own outputs (golden fixtures from
tests/golden/make_golden_3d.py), then the CUDA kernel through the C ABI
against the fixtures and the oracle.  Tolerance: 1e-5 relative L2 in fp32."""
import numpy as np
import pytest
import torch

from oracle import acoustic3d as o3
from oracle import oracle as orc

CASES = ["small_3d_nofs", "small_3d_fs"]
KEYS = ("p", "vx", "vy", "vz", "forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vy",
        "forward_wavefield_vz")


def load3(name):
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    with np.load(os.path.join(here, "golden", f"{name}.npz")) as z:
        c = {k: z[k] for k in z.files}
    for k in ("nz", "ny", "nx", "nabc", "nt"):
        c[k] = int(c[k])
    c["dx"], c["dt"], c["free_surface"] = float(c["dx"]), float(c["dt"]), bool(c["free_surface"])
    return c


def kw3(c):
    return dict(nz=c["nz"], ny=c["ny"], nx=c["nx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
                free_surface=c["free_surface"], src_x=c["src_x"], src_y=c["src_y"], src_z=c["src_z"],
                src_v=c["src_v"], rcv_x=c["rcv_x"], rcv_y=c["rcv_y"], rcv_z=c["rcv_z"], damp=c["damp"], vp=c["vp"],
                rho=c["rho"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_golden(name):
    c = load3(name)
    r64 = o3.forward(**kw3(c), dtype=np.float64)
    r32 = o3.forward(**kw3(c), dtype=np.float32)
    for k in KEYS:
        assert orc.rel_l2(r64[k], c[f"ref64_{k}"]) < 1e-12, k
        assert orc.rel_l2(r32[k], c[f"ref32_{k}"]) < 1e-6, k


def test_bc_pml_3d_matches_golden_damping():
    from geobrain_b200.wave import bc_pml_3d, create_boundary
    c = load3("small_3d_nofs")
    d = create_boundary("pml", nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], n_layers=c["nabc"],
                        vmax=float(c["vp"].max()), free_surface=False, ny=c["ny"], dy=c["dx"])
    np.testing.assert_array_equal(d.astype(np.float32), c["damp"])
    assert bc_pml_3d(16, 14, 12, 10.0, 10.0, 10.0, 6, 3000.0, free_surface=True).shape == (18, 26, 28)


def test_pad_model_3d_replicates_edges():
    from geobrain_b200.wave import pad_model_3d
    v = torch.arange(2 * 3 * 4, dtype=torch.float32).reshape(2, 3, 4)
    np.testing.assert_array_equal(pad_model_3d(v, 2, 2, 3, 4).numpy(), np.pad(v.numpy(), 2, mode="edge"))


def run3(c, device, **kw):
    from geobrain_b200.wave import acoustic_forward_kernel_3d
    out = acoustic_forward_kernel_3d(
        nx=c["nx"], ny=c["ny"], nz=c["nz"], dx=c["dx"], dy=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"],
        nabc=c["nabc"], free_surface=c["free_surface"], src_x=torch.as_tensor(c["src_x"]),
        src_y=torch.as_tensor(c["src_y"]), src_z=torch.as_tensor(c["src_z"]), src_n=len(c["src_x"]),
        src_v=torch.as_tensor(c["src_v"], device=device), rcv_x=torch.as_tensor(c["rcv_x"]),
        rcv_y=torch.as_tensor(c["rcv_y"]), rcv_z=torch.as_tensor(c["rcv_z"]), rcv_n=len(c["rcv_x"]),
        damp=torch.as_tensor(c["damp"], device=device), vp=torch.as_tensor(c["vp"], device=device),
        rho=torch.as_tensor(c["rho"], device=device), device=device, **kw)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_cuda_3d_matches_reference(cuda_device, name):
    c = load3(name)
    out = run3(c, cuda_device)
    for k in KEYS:
        assert orc.rel_l2(out[k], c[f"ref32_{k}"]) < 1e-5, (k, orc.rel_l2(out[k], c[f"ref32_{k}"]))
        assert orc.rel_l2(out[k], c[f"ref64_{k}"]) < 1e-5, k


@pytest.mark.gpu
def test_cuda_3d_larger_grid_against_oracle(cuda_device):
    """A ragged grid (sizes no multiple of the 128-column blocks) with more
    shots, a source in the padded border and receivers on the last valid
    planes, against the float64 oracle."""
    rng = np.random.default_rng(7)
    nz, ny, nx, nabc, nt = 23, 19, 61, 7, 60
    vp = (2000 + 800 * rng.random((nz, ny, nx))).astype(np.float32)
    rho = (1900 + 300 * rng.random((nz, ny, nx))).astype(np.float32)
    from geobrain_b200.wave import bc_pml_3d, RickerWavelet
    damp = bc_pml_3d(nx, ny, nz, 10.0, 10.0, 10.0, nabc, float(vp.max()), free_surface=False).astype(np.float32)
    w, _ = RickerWavelet()(f0=20.0, dt=1e-3)
    w = np.pad(w.numpy(), (0, nt))[:nt].astype(np.float32)
    c = dict(nz=nz, ny=ny, nx=nx, nabc=nabc, nt=nt, dx=10.0, dt=1e-3, free_surface=False, vp=vp, rho=rho,
             damp=damp, src_x=np.array([3, 30, -nabc, 50]), src_y=np.array([2, 9, -nabc, 17]),
             src_z=np.array([1, 11, -nabc, 20]), src_v=np.tile(w, (4, 1)),
             rcv_x=np.array([0, 10, 40, nx + nabc - 2, -nabc]), rcv_y=np.array([1, 5, 18, ny + nabc - 2, -nabc]),
             rcv_z=np.array([0, 3, 22, nz + nabc - 2, -nabc]))
    out = run3(c, cuda_device)
    ref = o3.forward(**kw3(c), dtype=np.float64)
    for k in KEYS:
        assert orc.rel_l2(out[k], ref[k]) < 1e-5, k


@pytest.mark.gpu
def test_cuda_3d_rejects_what_the_reference_cannot_index(cuda_device):
    c = load3("small_3d_nofs")
    bad = dict(c, rcv_x=np.array([c["nx"] + c["nabc"] - 1]), rcv_y=np.array([0]), rcv_z=np.array([0]))
    with pytest.raises(ValueError):
        run3(bad, cuda_device)
    with pytest.raises(ValueError):
        run3(dict(c, src_z=np.array([c["nz"] + c["nabc"], 0])), cuda_device)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("segments,imaging_cache", [(1, 0), (4, 0), (1, "auto")])
def test_cuda_3d_gradient_matches_reference_autograd(cuda_device, name, segments, imaging_cache):
    """dL/dvp and dL/drho of a loss linear in all four traces: the
    hand-written 3-D adjoint (checkpointed recompute, or every step's imaging
    fields kept by the forward) against the reference's float64 autograd
    gradient, 1e-4 relative L2."""
    from geobrain_b200.wave import acoustic_forward_kernel_3d
    c = load3(name)
    vp = torch.tensor(c["vp"], device=cuda_device, requires_grad=True)
    rho = torch.tensor(c["rho"], device=cuda_device, requires_grad=True)
    out = acoustic_forward_kernel_3d(
        nx=c["nx"], ny=c["ny"], nz=c["nz"], dx=c["dx"], dy=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"],
        nabc=c["nabc"], free_surface=c["free_surface"], src_x=c["src_x"], src_y=c["src_y"], src_z=c["src_z"],
        src_n=2, src_v=torch.as_tensor(c["src_v"], device=cuda_device), rcv_x=c["rcv_x"], rcv_y=c["rcv_y"],
        rcv_z=c["rcv_z"], rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=cuda_device), vp=vp,
        rho=rho, checkpoint_segments=segments, device=cuda_device, imaging_cache=imaging_cache)
    loss = sum((torch.as_tensor(c[f"lin_{k}"], device=cuda_device, dtype=torch.float32) * out[k]).sum()
               for k in ("p", "vx", "vy", "vz"))
    loss.backward()
    assert orc.rel_l2(vp.grad.cpu().numpy(), c["ref64_grad_vp"]) < 1e-4
    assert orc.rel_l2(rho.grad.cpu().numpy(), c["ref64_grad_rho"]) < 1e-4


@pytest.mark.gpu
def test_cuda_3d_imaging_cache_and_recompute_agree(cuda_device):
    """Velocity-only and velocity + density gradients through both storage
    modes: the cached imaging fields are the numbers the recompute writes,
    so the two gradients are identical."""
    from geobrain_b200.wave import acoustic_forward_kernel_3d
    c = load3("small_3d_fs")
    for want_rho in (False, True):
        grads = []
        for cache in (0, "auto"):
            vp = torch.tensor(c["vp"], device=cuda_device, requires_grad=True)
            rho = torch.tensor(c["rho"], device=cuda_device, requires_grad=want_rho)
            out = acoustic_forward_kernel_3d(
                nx=c["nx"], ny=c["ny"], nz=c["nz"], dx=c["dx"], dy=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"],
                nabc=c["nabc"], free_surface=c["free_surface"], src_x=c["src_x"], src_y=c["src_y"],
                src_z=c["src_z"], src_n=2, src_v=torch.as_tensor(c["src_v"], device=cuda_device), rcv_x=c["rcv_x"],
                rcv_y=c["rcv_y"], rcv_z=c["rcv_z"], rcv_n=len(c["rcv_x"]),
                damp=torch.as_tensor(c["damp"], device=cuda_device), vp=vp, rho=rho, device=cuda_device,
                imaging_cache=cache)
            (0.5 * (out["p"] ** 2).sum() + out["vz"].sum()).backward()
            grads.append((vp.grad.cpu().numpy(), rho.grad.cpu().numpy() if want_rho else None))
        np.testing.assert_array_equal(grads[0][0], grads[1][0])
        if want_rho:
            np.testing.assert_array_equal(grads[0][1], grads[1][1])


def test_oracle_gradient_matches_reference_autograd():
    for name in CASES:
        c = load3(name)
        gv, gr = o3.gradient(**kw3(c), res_p=c["lin_p"], res_vx=c["lin_vx"], res_vy=c["lin_vy"],
                             res_vz=c["lin_vz"])
        assert orc.rel_l2(gv, c["ref64_grad_vp"]) < 1e-12
        assert orc.rel_l2(gr, c["ref64_grad_rho"]) < 1e-12


@pytest.mark.gpu
def test_propagator_runs_3d_models(cuda_device):
    """AcousticPropagator on a 3-D AcousticModel and Survey dispatches to the
    3-D kernel (propagators/acoustic.py:220-247), with the survey's (x, y, z)
    locations."""
    from geobrain_b200.wave import (AcousticModel, AcousticPropagator, BoundaryConfig, GridConfig, Receiver,
                                    Source, Survey)
    c = load3("small_3d_nofs")
    grid = GridConfig(nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], ny=c["ny"], dy=c["dx"])
    model = AcousticModel(grid, BoundaryConfig(n_layers=c["nabc"]), vp=c["vp"], rho=c["rho"], auto_update_rho=False,
                          device=str(cuda_device))
    src = Source(nt=c["nt"], dt=c["dt"], f0=25.0)
    src.add_sources(x=c["src_x"], z=c["src_z"], y=c["src_y"], wavelet=c["src_v"][0])
    rcv = Receiver(nt=c["nt"], dt=c["dt"])
    rcv.add_receivers(x=c["rcv_x"], z=c["rcv_z"], y=c["rcv_y"], rcv_type="pr")
    prop = AcousticPropagator(model, Survey(src, rcv), device=str(cuda_device))
    res = prop.forward()
    assert res.vy is not None
    for k in ("p", "vx", "vy", "vz"):
        assert orc.rel_l2(getattr(res, k).cpu().numpy(), c[f"ref32_{k}"]) < 1e-5, k


def test_oracle_wavelet_gradient_is_exact_for_the_linear_source():
    """The traces are linear in the wavelet, so <dL/dw, d> equals
    (L(w + d) - L(w - d)) / 2 up to rounding, for any d."""
    c = load3("small_3d_fs")
    lin = {k: c[f"lin_{k}"] for k in ("p", "vx", "vy", "vz")}
    _, _, gw = o3.gradient(**kw3(c), res_p=lin["p"], res_vx=lin["vx"], res_vy=lin["vy"], res_vz=lin["vz"],
                           with_wavelet=True)
    d = np.random.default_rng(4).standard_normal(c["src_v"].shape)

    def loss(w):
        out = o3.forward(**dict(kw3(c), src_v=w), dtype=np.float64)
        return sum(float((lin[k] * out[k]).sum()) for k in lin)

    w0 = c["src_v"].astype(np.float64)
    fd = (loss(w0 + d) - loss(w0 - d)) / 2
    assert abs(fd - float((gw * d).sum())) <= 1e-10 * abs(fd)


@pytest.mark.gpu
@pytest.mark.parametrize("imaging_cache", [0, "auto"])
def test_cuda_3d_wavelet_gradient_matches_oracle(cuda_device, imaging_cache):
    """dL/d(src_v) with the model gradient, a source on the outermost padded
    plane included (the 3-D adjoint keeps lambda everywhere)."""
    from geobrain_b200.wave import acoustic_forward_kernel_3d
    c = dict(load3("small_3d_fs"))
    c["src_x"] = np.array([c["src_x"][0], -c["nabc"]])
    lin = {k: c[f"lin_{k}"] for k in ("p", "vx", "vy", "vz")}
    w = torch.tensor(c["src_v"], device=cuda_device, requires_grad=True)
    vp = torch.tensor(c["vp"], device=cuda_device, requires_grad=True)
    out = acoustic_forward_kernel_3d(
        nx=c["nx"], ny=c["ny"], nz=c["nz"], dx=c["dx"], dy=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"],
        nabc=c["nabc"], free_surface=c["free_surface"], src_x=c["src_x"], src_y=c["src_y"], src_z=c["src_z"],
        src_n=2, src_v=w, rcv_x=c["rcv_x"], rcv_y=c["rcv_y"], rcv_z=c["rcv_z"], rcv_n=len(c["rcv_x"]),
        damp=torch.as_tensor(c["damp"], device=cuda_device), vp=vp,
        rho=torch.as_tensor(c["rho"], device=cuda_device), device=cuda_device, imaging_cache=imaging_cache)
    sum((torch.as_tensor(lin[k], device=cuda_device, dtype=torch.float32) * out[k]).sum() for k in lin).backward()
    rvp, _, rw = o3.gradient(**kw3(c), res_p=lin["p"], res_vx=lin["vx"], res_vy=lin["vy"], res_vz=lin["vz"],
                             with_wavelet=True)
    assert orc.rel_l2(w.grad.cpu().numpy(), rw) < 1e-4, orc.rel_l2(w.grad.cpu().numpy(), rw)
    assert orc.rel_l2(vp.grad.cpu().numpy(), rvp) < 1e-4


def _fused_vs_split_case(shots, free_surface, nz=23, ny=19, nx=121, nabc=7, nt=40, seed=11):
    rng = np.random.default_rng(seed)
    vp = (2000 + 800 * rng.random((nz, ny, nx))).astype(np.float32)
    rho = (1900 + 300 * rng.random((nz, ny, nx))).astype(np.float32)
    from geobrain_b200.wave import bc_pml_3d, RickerWavelet
    # the full padded damping (the 3-D entry point takes it whether or not the top is a free surface)
    damp = bc_pml_3d(nx, ny, nz, 10.0, 10.0, 10.0, nabc, float(vp.max()), free_surface=False).astype(np.float32)
    w, _ = RickerWavelet()(f0=20.0, dt=1e-3)
    w = np.pad(w.numpy(), (0, nt))[:nt].astype(np.float32)
    # sources: a grid corner, the last column of an x tile (padded 119), the padded border, then random
    sx = np.concatenate([[-nabc, 119 - nabc, nx + nabc - 1], rng.integers(0, nx, shots)])[:shots]
    sy = np.concatenate([[-nabc, 5, ny + nabc - 1], rng.integers(0, ny, shots)])[:shots]
    sz = np.concatenate([[-nabc, 0, nz + nabc - 1], rng.integers(0, nz, shots)])[:shots]
    return dict(nz=nz, ny=ny, nx=nx, nabc=nabc, nt=nt, dx=10.0, dt=1e-3, free_surface=free_surface, vp=vp,
                rho=rho, damp=damp, src_x=sx, src_y=sy, src_z=sz, src_v=np.tile(w, (shots, 1)),
                rcv_x=np.arange(0, nx, 3), rcv_y=np.full(len(range(0, nx, 3)), ny // 2),
                rcv_z=np.full(len(range(0, nx, 3)), 3))   # below the free surface, where p is not 0


def _with_step_kernel(mode, fn):
    from geobrain_b200 import _lib
    L = _lib.load()
    prev = L.gb3_set_fused_step(int(mode))
    try:
        return fn()
    finally:
        L.gb3_set_fused_step(prev)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("shots", [3, 10])
@pytest.mark.parametrize("free_surface", [False, True])
def test_cuda_3d_fused_step_equals_split_kernels(cuda_device, mode, shots, free_surface):
    """The fused step (one z-marching launch per step, csrc/gb_3d_fused.cuh;
    mode 1: 8-row tiles, mode 2: 16-row tiles) against the split pressure /
    velocity kernels on a grid of 2 x 5 (2 x 3) tiles
    with ragged edges and sources on tile and grid borders: traces and both
    gradients (recompute from checkpoints, and the imaging cache with the
    density) bit-identical.  Energies: identical up to 8 shots (one cluster
    adds its shots in order, as the split kernels' shot loop); above 8 the
    clusters add to the maps one after another, within 1e-6."""
    from geobrain_b200.wave import acoustic_forward_kernel_3d
    c = _fused_vs_split_case(shots, free_surface)

    def run():
        out = run3(c, cuda_device)
        grads = []
        for segments, cache in ((3, 0), (1, "auto")):
            vp = torch.tensor(c["vp"], device=cuda_device, requires_grad=True)
            rho = torch.tensor(c["rho"], device=cuda_device, requires_grad=True)
            o = acoustic_forward_kernel_3d(
                nx=c["nx"], ny=c["ny"], nz=c["nz"], dx=c["dx"], dy=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"],
                nabc=c["nabc"], free_surface=c["free_surface"], src_x=c["src_x"], src_y=c["src_y"],
                src_z=c["src_z"], src_n=shots, src_v=torch.as_tensor(c["src_v"], device=cuda_device),
                rcv_x=c["rcv_x"], rcv_y=c["rcv_y"], rcv_z=c["rcv_z"], rcv_n=len(c["rcv_x"]),
                damp=torch.as_tensor(c["damp"], device=cuda_device), vp=vp, rho=rho,
                checkpoint_segments=segments, device=cuda_device, imaging_cache=cache)
            (0.5 * (o["p"] ** 2).sum() + o["vx"].sum() - o["vy"].sum() + o["vz"].sum()).backward()
            grads.append((vp.grad.cpu().numpy(), rho.grad.cpu().numpy()))
        return out, grads

    split, g_split = _with_step_kernel(0, run)
    fused, g_fused = _with_step_kernel(mode, run)
    for k in ("p", "vx", "vy", "vz"):
        np.testing.assert_array_equal(fused[k], split[k], err_msg=k)
    for k in KEYS[4:]:
        if shots <= 8:
            np.testing.assert_array_equal(fused[k], split[k], err_msg=k)
        else:
            assert orc.rel_l2(fused[k], split[k]) < 1e-6, k
    assert np.abs(fused["p"]).max() > 0
    for (gv_s, gr_s), (gv_f, gr_f) in zip(g_split, g_fused):
        np.testing.assert_array_equal(gv_f, gv_s)
        np.testing.assert_array_equal(gr_f, gr_s)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [1, 2])
def test_cuda_3d_fused_step_at_the_benchmark_size(cuda_device, mode):
    """The 200^3 + 20-cell PML model with 4 shots (the 3-D rate workload),
    20 steps: traces and energies of the fused step equal the split kernels'
    bit for bit."""
    rng = np.random.default_rng(0)
    nz = ny = nx = 200
    nabc, nt, shots = 20, 20, 4
    from geobrain_b200.wave import bc_pml_3d, RickerWavelet
    vp = (2000 + 1000 * rng.random((nz, ny, nx))).astype(np.float32)
    w, _ = RickerWavelet()(f0=15.0, dt=1e-3)
    w = np.pad(w.numpy(), (0, nt))[:nt].astype(np.float32)
    c = dict(nz=nz, ny=ny, nx=nx, nabc=nabc, nt=nt, dx=10.0, dt=1e-3, free_surface=False, vp=vp,
             rho=np.full((nz, ny, nx), 2000.0, np.float32),
             damp=bc_pml_3d(nx, ny, nz, 10.0, 10.0, 10.0, nabc, 3000.0, free_surface=False).astype(np.float32),
             src_x=np.linspace(10, nx - 10, shots).astype(np.int64), src_y=np.full(shots, ny // 2),
             src_z=np.ones(shots, np.int64), src_v=np.tile(w, (shots, 1)), rcv_x=np.arange(0, nx, 2),
             rcv_y=np.full(nx // 2, ny // 2), rcv_z=np.ones(nx // 2, np.int64))
    split = _with_step_kernel(0, lambda: run3(c, cuda_device))
    fused = _with_step_kernel(mode, lambda: run3(c, cuda_device))
    for k in KEYS:
        np.testing.assert_array_equal(fused[k], split[k], err_msg=k)
    assert np.abs(fused["p"]).max() > 0
