"""gb_forward_static_scratch: forward modelling for callers that cannot
allocate device memory (their host's memory pool owns the GPU), with the
library's scratch in a fixed 64 MiB static device array instead of a
workspace.  Checked through the C ABI against gb_forward on the same inputs,
on two calls in a row (the second call must not see the first call's
leftovers in the shared array).  Collected last on purpose."""
import numpy as np
import pytest
import torch

from conftest import load_case
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _inputs(c, dev, fd_order):
    from geobrain_b200.wave import engine
    geo = engine.Geometry(c["nz"], c["nx"], c["nabc"], c["nt"], c["dt"], c["dx"], fd_order // 2,
                          c["free_surface"])
    plan = engine.get_plan(geo, c["src_x"], c["src_z"], c["rcv_x"], c["rcv_z"])
    t = {k: torch.tensor(c[k], dtype=torch.float32, device=dev).contiguous()
         for k in ("vp", "rho", "damp", "src_v")}
    return plan, t


def _static_call(plan, t, dev):
    lib = plan._lib
    S, NR, nt = plan.n_shots, plan.n_rcv, plan.geo.nt
    nz, nx = plan.geo.nz, plan.geo.nx
    tr = [torch.full((S, nt, NR), float("nan"), device=dev) for _ in range(3)]
    en = [torch.full((nz, nx), float("nan"), device=dev) for _ in range(3)]
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.gb_forward_static_scratch(plan.h, t["vp"].data_ptr(), t["rho"].data_ptr(), t["damp"].data_ptr(),
                                       t["src_v"].data_ptr(), *[x.data_ptr() for x in tr],
                                       *[x.data_ptr() for x in en], 0, None, stream)
    assert rc == 0, lib.gb_last_error()
    torch.cuda.synchronize()
    return [x.cpu().numpy() for x in tr], [x.cpu().numpy() for x in en]


@pytest.mark.parametrize("name,fd_order", [("small_fs", 4), ("layered_100x200", 8)])
def test_static_scratch_matches_workspace_forward(cuda_device, name, fd_order):
    from geobrain_b200.wave import engine
    c = load_case(name)
    plan, t = _inputs(c, cuda_device, fd_order)
    ref = engine.run_forward(plan, t["vp"], t["rho"], t["damp"], t["src_v"], want_energy=True)
    ref_tr = [x.cpu().numpy() for x in ref[:3]]
    ref_en = [x.cpu().numpy() for x in ref[3]]
    for _ in range(2):
        tr, en = _static_call(plan, t, cuda_device)
        for a, b in zip(tr, ref_tr):
            assert orc.rel_l2(a, b) < TOL
        for a, b in zip(en, ref_en):
            assert orc.rel_l2(a, b) < TOL


def test_static_scratch_rejects_models_beyond_its_size(cuda_device):
    from geobrain_b200.wave import engine
    lib = engine._lib.load()
    limit = lib.gb_static_scratch_bytes()
    assert limit == 64 << 20
    nz, nx, nabc = 1000, 3000, 40
    geo = engine.Geometry(nz, nx, nabc, 10, 4e-4, 5.0, 4, False)
    plan = engine.get_plan(geo, np.array([10, 20]), np.array([1, 1]), np.arange(5), np.ones(5, np.int64))
    assert plan.workspace_bytes(False, 0) > limit
    z = torch.zeros(1, device=cuda_device)
    rc = lib.gb_forward_static_scratch(plan.h, z.data_ptr(), z.data_ptr(), z.data_ptr(), z.data_ptr(), None, None,
                                       None, None, None, None, 0, None, torch.cuda.current_stream().cuda_stream)
    assert rc == -3
    assert b"static scratch" in lib.gb_last_error()


@pytest.mark.parametrize("name,fd_order", [("small_nofs", 8), ("small_fs", 4)])
def test_static_scratch_with_cpml_layers(cuda_device, name, fd_order):
    """A CPML plan (its memory variables live in the same scratch) through
    the no-alloc entry point: the same outputs as the workspace forward, on
    two calls in a row (the memory variables restart from zero each call)."""
    from geobrain_b200.wave import engine
    c = load_case(name)
    plan, t = _inputs(c, cuda_device, fd_order)
    try:
        plan.set_absorbing("cpml", float(c["vp"].max()))
        ref = engine.run_forward(plan, t["vp"], t["rho"], t["damp"], t["src_v"], want_energy=True)
        ref_tr = [x.cpu().numpy() for x in ref[:3]]
        ref_en = [x.cpu().numpy() for x in ref[3]]
        for _ in range(2):
            tr, en = _static_call(plan, t, cuda_device)
            for a, b in zip(tr + en, ref_tr + ref_en):
                assert orc.rel_l2(a, b) < TOL
    finally:
        plan.set_absorbing("damping")
