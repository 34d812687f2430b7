"""Gradient parity of the hand-written adjoint (through the C ABI) against the
reference's float64 autograd gradient (golden fixtures), the float64 CPU
oracle for the 8th-order scheme, and central finite differences.

Tolerance: 1e-4 relative L2 against float64 (the float32 restatement itself
sits near 2e-6; the bar set for the propagator is 1e-3)."""
import numpy as np
import pytest
import torch

from conftest import load_case, oracle_kwargs
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
GTOL = 1e-4


def cuda_grad(c, device, fd_order=4, lin=None, want_rho=True, **kw):
    from geobrain_b200.wave import acoustic_forward_kernel
    S = len(c["src_x"])
    vp = torch.tensor(c["vp"], device=device, requires_grad=True)
    rho = torch.tensor(c["rho"], device=device, requires_grad=want_rho)
    out = acoustic_forward_kernel(
        nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
        free_surface=c["free_surface"], src_x=c["src_x"], src_z=c["src_z"], src_n=S,
        src_v=torch.as_tensor(c["src_v"], device=device), rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
        rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=device), vp=vp, rho=rho, device=device,
        fd_order=fd_order, **kw)
    lin = lin if lin is not None else {k: c[f"lin_{k}"] for k in ("p", "vx", "vz")}
    loss = sum((torch.as_tensor(lin[k], device=device, dtype=torch.float32) * out[k]).sum()
               for k in ("p", "vx", "vz") if lin.get(k) is not None)
    loss.backward()
    torch.cuda.synchronize()
    return vp.grad.cpu().numpy(), (rho.grad.cpu().numpy() if want_rho else None), float(loss.detach())


@pytest.mark.parametrize("name", ["small_nofs", "small_fs"])
def test_gradient_matches_reference_autograd(cuda_device, name):
    c = load_case(name)
    gvp, grho, _ = cuda_grad(c, cuda_device, checkpoint_segments=3)
    assert orc.rel_l2(gvp, c["ref64_grad_vp"]) < GTOL
    assert orc.rel_l2(grho, c["ref64_grad_rho"]) < GTOL


@pytest.mark.parametrize("name", ["small_nofs", "small_fs"])
def test_eighth_order_gradient_matches_oracle(cuda_device, name):
    c = load_case(name)
    gvp, grho, _ = cuda_grad(c, cuda_device, fd_order=8)
    rvp, rrho, _ = orc.gradient(**oracle_kwargs(c), res_p=c["lin_p"], res_vx=c["lin_vx"], res_vz=c["lin_vz"],
                                half=4, dtype=np.float64)
    assert orc.rel_l2(gvp, rvp) < GTOL
    assert orc.rel_l2(grho, rrho) < GTOL


@pytest.mark.parametrize("imaging_cache", [0, "auto", "partial"])
def test_segment_length_and_cache_do_not_change_gradient(cuda_device, imaging_cache):
    """fp32 checkpoints restart the recompute bit for bit, and cached imaging
    fields are the same numbers the recompute writes, so every segment length
    and cache size gives the identical gradient."""
    c = load_case("small_nofs")
    base, _, _ = cuda_grad(c, cuda_device, fd_order=8, want_rho=False, checkpoint_every=c["nt"], imaging_cache=0)
    if imaging_cache == "partial":
        from geobrain_b200.wave import engine
        geo = engine.Geometry(c["nz"], c["nx"], c["nabc"], c["nt"], c["dt"], c["dx"], 4, False)
        plan = engine.get_plan(geo, c["src_x"], c["src_z"], c["rcv_x"], c["rcv_z"])
        imaging_cache = plan.imaging_bytes(c["nt"] // 3 + 5, False)      # a third of the steps, off-segment
    for k in (1, 7, 64):
        g, _, _ = cuda_grad(c, cuda_device, fd_order=8, want_rho=False, checkpoint_every=k,
                            imaging_cache=imaging_cache)
        np.testing.assert_array_equal(g, base)


def test_group_streams_do_not_change_results(cuda_device):
    from geobrain_b200.wave import engine
    c = load_case("small_fs")
    geo = engine.Geometry(c["nz"], c["nx"], c["nabc"], c["nt"], c["dt"], c["dx"], 2, True)
    plan = engine.get_plan(geo, c["src_x"], c["src_z"], c["rcv_x"], c["rcv_z"])
    plan.set_tiling(16, 1)                 # three groups of one shot
    try:
        a = cuda_grad(c, cuda_device, imaging_cache=0, checkpoint_every=50)
        plan.set_group_streams(False)
        b = cuda_grad(c, cuda_device, imaging_cache=0, checkpoint_every=50)
    finally:
        plan.set_group_streams(True)
        plan.set_tiling(16, 0)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert a[2] == b[2]


@pytest.mark.parametrize("imaging_cache", [0, "auto"])
def test_cta_schedule_does_not_change_gradient(cuda_device, imaging_cache):
    """The guided CTA order against blockIdx order: the gradients and the
    loss bit for bit (each (group, cell) gradient sum keeps one owner and
    its time order)."""
    from geobrain_b200.wave import engine
    c = load_case("small_fs")
    geo = engine.Geometry(c["nz"], c["nx"], c["nabc"], c["nt"], c["dt"], c["dx"], 2, True)
    plan = engine.get_plan(geo, c["src_x"], c["src_z"], c["rcv_x"], c["rcv_z"])
    plan.set_tiling(16, 1)                 # three groups of one shot
    try:
        plan.set_schedule(0)
        a = cuda_grad(c, cuda_device, imaging_cache=imaging_cache, checkpoint_every=50)
        plan.set_schedule(1)
        b = cuda_grad(c, cuda_device, imaging_cache=imaging_cache, checkpoint_every=50)
    finally:
        plan.set_schedule(0)
        plan.set_tiling(16, 0)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert a[2] == b[2]


@pytest.mark.parametrize("fmt,every,tol", [("fp24", 10, GTOL), ("fp24", 20, GTOL), ("fp16", 20, 1e-3),
                                           ("bf16", 20, 1e-2)])
def test_short_checkpoints_within_budget(cuda_device, fmt, every, tol):
    """Snapshots stored in 24 bits (fp32 exponent, 15-bit mantissa) or in 16
    bits with a per-snapshot scale; the recompute from them runs in fp32, so
    the only error is each segment restarting from a rounded state (12 or 24
    restarts here, the harshest cases).  fp24 keeps 16 significant bits and
    stays at the fp32 bar; fp16 keeps 11 (about 6e-4 here), bf16 8 (about 8x
    more than fp16)."""
    c = load_case("small_nofs")
    g, _, _ = cuda_grad(c, cuda_device, fd_order=8, want_rho=False, checkpoint_every=every, imaging_cache=0,
                        snapshot_dtype=fmt)
    rvp, _, _ = orc.gradient(**oracle_kwargs(c), res_p=c["lin_p"], res_vx=c["lin_vx"], res_vz=c["lin_vz"],
                             half=4, dtype=np.float64)
    err = orc.rel_l2(g, rvp)
    assert err < tol, err


@pytest.mark.parametrize("fmt,tol", [("fp24", GTOL), ("bf16", 1e-2)])
@pytest.mark.parametrize("cache,want_rho", [("auto", False), ("partial", False), ("auto", True)])
def test_short_imaging_cache_within_budget(cuda_device, fmt, tol, cache, want_rho):
    """Imaging fields cached in 24 or 16 bits: each is rounded once
    (relative 2^-16 or 2^-9) and enters the gradient sums once, without
    passing through the wave equation; the sums cancel, so the gradient's
    error is of the order of the format's precision (fp24 keeps the fp32
    bar; bf16 measures about 3e-3).  'partial' mixes cached steps with fp32
    recomputed segments."""
    c = load_case("small_nofs")
    if cache == "partial":
        from geobrain_b200.wave import engine
        geo = engine.Geometry(c["nz"], c["nx"], c["nabc"], c["nt"], c["dt"], c["dx"], 4, False)
        plan = engine.get_plan(geo, c["src_x"], c["src_z"], c["rcv_x"], c["rcv_z"])
        cache = plan.imaging_bytes(c["nt"] // 2 + 3, want_rho, fmt)
    gvp, grho, _ = cuda_grad(c, cuda_device, fd_order=8, want_rho=want_rho, checkpoint_every=16,
                             imaging_cache=cache, imaging_dtype=fmt)
    rvp, rrho, _ = orc.gradient(**oracle_kwargs(c), res_p=c["lin_p"], res_vx=c["lin_vx"], res_vz=c["lin_vz"],
                                half=4, dtype=np.float64)
    err = orc.rel_l2(gvp, rvp)
    assert err < tol, err
    if want_rho:
        assert orc.rel_l2(grho, rrho) < tol
    g32, _, _ = cuda_grad(c, cuda_device, fd_order=8, want_rho=want_rho, checkpoint_every=16, imaging_cache=0)
    assert orc.rel_l2(gvp, g32) < tol
    assert not np.array_equal(gvp, g32)          # the cached steps really came from the short store


def test_shot_subsets_sum_to_the_full_gradient(cuda_device):
    """The rank-local FWI function of the sharded path: gradients of shot
    subsets add up to the all-shot gradient (the split changes only the
    order of the fp32 sums)."""
    from geobrain_b200.wave import sharding
    c = load_case("small_nofs")
    kk = dict(nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
              free_surface=False, src_x=c["src_x"], src_z=c["src_z"], src_n=3,
              src_v=torch.as_tensor(c["src_v"], device=cuda_device), rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
              rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=cuda_device), device=cuda_device,
              fd_order=8)
    vp = torch.tensor(c["vp"], device=cuda_device)
    rho = torch.tensor(c["rho"], device=cuda_device)
    d_obs = torch.tensor(c["ref32_p"] * 0.9, device=cuda_device)
    run = sharding.fwi_local_fn(kk, vp, rho, d_obs)
    l_all, g_all = run([0, 1, 2])
    l_a, g_a = run([0, 2])
    l_b, g_b = run([1])
    assert abs(float(l_a + l_b) - float(l_all)) <= 1e-5 * abs(float(l_all))
    assert orc.rel_l2((g_a + g_b).cpu().numpy(), g_all.cpu().numpy()) < 1e-6
    l_s, g_s = sharding.sharded_shot_gradient(3, run)          # one process: one call over all shots
    np.testing.assert_array_equal(g_s.cpu().numpy(), g_all.cpu().numpy())
    z_l, z_g = run([])
    assert float(z_l) == 0.0 and not z_g.any()


@pytest.mark.parametrize("want_rho", [False, True])
def test_streaming_recompute_is_bit_identical(cuda_device, want_rho):
    """Recompute segments (and the forward) through the streaming kernel
    write the same imaging fields, so the gradient is bit-identical."""
    from geobrain_b200.wave import engine
    c = load_case("small_nofs")
    geo = engine.Geometry(c["nz"], c["nx"], c["nabc"], c["nt"], c["dt"], c["dx"], 4, False)
    plan = engine.get_plan(geo, c["src_x"], c["src_z"], c["rcv_x"], c["rcv_z"])
    base = cuda_grad(c, cuda_device, fd_order=8, want_rho=want_rho, checkpoint_every=17, imaging_cache=0)
    plan.set_streaming(True, 2)
    try:
        got = cuda_grad(c, cuda_device, fd_order=8, want_rho=want_rho, checkpoint_every=17, imaging_cache=0)
    finally:
        plan.set_streaming(False)
    np.testing.assert_array_equal(got[0], base[0])
    if want_rho:
        np.testing.assert_array_equal(got[1], base[1])


def test_velocity_only_gradient_matches_full(cuda_device):
    c = load_case("small_fs")
    g1, _, _ = cuda_grad(c, cuda_device, want_rho=False)
    g2, _, _ = cuda_grad(c, cuda_device, want_rho=True)
    assert orc.rel_l2(g1, g2) < 1e-6


def test_pressure_only_residual(cuda_device):
    """An L2 misfit on pressure traces only (vx / vz receive no gradient)."""
    c = load_case("small_nofs")
    lin = {"p": c["lin_p"], "vx": None, "vz": None}
    gvp, _, _ = cuda_grad(c, cuda_device, fd_order=8, lin=lin, want_rho=False)
    rvp, _, _ = orc.gradient(**oracle_kwargs(c), res_p=c["lin_p"], half=4, dtype=np.float64)
    assert orc.rel_l2(gvp, rvp) < GTOL


def test_gradient_central_difference(cuda_device):
    """Directional derivative of an L2 misfit on the CUDA forward itself."""
    from geobrain_b200.wave import acoustic_forward_kernel
    c = load_case("small_nofs")
    rng = np.random.default_rng(0)
    d_obs = torch.tensor(c["ref32_p"] * 0.9, device=cuda_device)

    def loss_at(vp_np, grad=False):
        vp = torch.tensor(vp_np, device=cuda_device, requires_grad=grad)
        out = acoustic_forward_kernel(
            nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
            free_surface=False, src_x=c["src_x"], src_z=c["src_z"], src_n=3,
            src_v=torch.as_tensor(c["src_v"], device=cuda_device), rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
            rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=cuda_device), vp=vp,
            rho=torch.as_tensor(c["rho"], device=cuda_device), device=cuda_device, fd_order=8)
        loss = 0.5 * ((out["p"].double() - d_obs.double()) ** 2).sum()
        if grad:
            loss.backward()
            return float(loss.detach()), vp.grad.cpu().numpy().astype(np.float64)
        return float(loss)

    _, g = loss_at(c["vp"], grad=True)
    dv = rng.standard_normal(c["vp"].shape).astype(np.float32) * 5.0
    fd = (loss_at(c["vp"] + dv) - loss_at(c["vp"] - dv)) / 2.0
    an = float(np.sum(g * dv))
    assert abs(fd - an) <= 2e-3 * abs(an), (fd, an)


def _wavelet_run(c, device, fd_order, model_grad, **kw):
    from geobrain_b200.wave import acoustic_forward_kernel
    w = torch.tensor(c["src_v"], device=device, requires_grad=True)
    vp = torch.tensor(c["vp"], device=device, requires_grad=model_grad)
    out = acoustic_forward_kernel(
        nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
        free_surface=c["free_surface"], src_x=c["src_x"], src_z=c["src_z"], src_n=len(c["src_x"]), src_v=w,
        rcv_x=c["rcv_x"], rcv_z=c["rcv_z"], rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=device),
        vp=vp, rho=torch.as_tensor(c["rho"], device=device), device=device, fd_order=fd_order, **kw)
    loss = sum((torch.as_tensor(c[f"lin_{k}"], device=device, dtype=torch.float32) * out[k]).sum()
               for k in ("p", "vx", "vz"))
    loss.backward()
    return w.grad.cpu().numpy(), (vp.grad.cpu().numpy() if model_grad else None)


@pytest.mark.parametrize("name", ["small_nofs", "small_fs"])
@pytest.mark.parametrize("fd_order", [4, 8])
@pytest.mark.parametrize("model_grad", [True, False])
def test_wavelet_gradient_matches_oracle(cuda_device, name, fd_order, model_grad):
    """dL/d(src_v), what autograd through the reference's source injection
    (acoustic_2d.py:228-237) gives, against the float64 oracle; with and
    without the model gradient in the same backward."""
    c = load_case(name)
    gw, gvp = _wavelet_run(c, cuda_device, fd_order, model_grad, checkpoint_segments=3)
    rvp, _, rw = orc.gradient(**oracle_kwargs(c), res_p=c["lin_p"], res_vx=c["lin_vx"], res_vz=c["lin_vz"],
                              half=fd_order // 2, dtype=np.float64)
    assert orc.rel_l2(gw, rw) < GTOL, orc.rel_l2(gw, rw)
    if model_grad:
        assert orc.rel_l2(gvp, rvp) < GTOL


def test_wavelet_gradient_refuses_sources_outside_the_update_region(cuda_device):
    c = load_case("small_nofs")
    c = dict(c, src_z=np.array([1, 1, -c["nabc"]]))          # the last shot on the outermost padded row
    with pytest.raises(NotImplementedError):
        _wavelet_run(c, cuda_device, 4, False)


@pytest.mark.parametrize("nabc", [12, 16])
def test_gradient_with_receivers_above_the_free_surface(cuda_device, nabc):
    """Receivers in rows fs-1, fs and fs+1 under a free surface, a loss linear
    in all three traces: the vz trace in row fs-1 is vz[fs] after the mirror,
    so its adjoint source lands in row fs.  Against the float64 oracle; with
    nabc = 16 the surface falls on a 16-row tile edge."""
    from test_forward_gpu import synthetic_case
    c = dict(synthetic_case(50, 200, nabc, 150, 2, seed=9), free_surface=True)
    rx = np.arange(0, 200, 7)
    c["rcv_x"] = np.concatenate([rx, rx, rx])
    c["rcv_z"] = np.concatenate([np.full(rx.size, -1), np.zeros(rx.size, np.int64), np.ones(rx.size, np.int64)])
    c["src_z"], c["src_x"] = np.array([2, 5]), np.array([40, 150])
    rng = np.random.default_rng(10)
    lin = {k: rng.standard_normal((2, 150, c["rcv_x"].size)) for k in ("p", "vx", "vz")}
    gvp, grho, _ = cuda_grad(c, cuda_device, fd_order=8, lin=lin)
    rvp, rrho, _ = orc.gradient(**oracle_kwargs(c), res_p=lin["p"], res_vx=lin["vx"], res_vz=lin["vz"], half=4,
                                dtype=np.float64)
    assert orc.rel_l2(gvp, rvp) < GTOL
    assert orc.rel_l2(grho, rrho) < GTOL
