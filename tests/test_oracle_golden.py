"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the GeoBrain PyTorch path).  CPU only."""
import numpy as np
import pytest

from conftest import load_case, oracle_kwargs
from oracle import oracle as orc

CASES = ["small_nofs", "small_fs"]


@pytest.mark.parametrize("name", CASES)
def test_fp64_forward_matches_reference_fp64(name):
    c = load_case(name)
    out = orc.forward(**oracle_kwargs(c), dtype=np.float64)
    for k in ("p", "vx", "vz", "forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        assert orc.rel_l2(out[k], c[f"ref64_{k}"]) < 1e-12, k


@pytest.mark.parametrize("name", CASES)
def test_fp32_forward_matches_reference_fp32(name):
    c = load_case(name)
    out = orc.forward(**oracle_kwargs(c), dtype=np.float32, snapshot_every=int(c["snapshot_every"]))
    for k in ("p", "vx", "vz", "forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        assert orc.rel_l2(out[k], c[f"ref32_{k}"]) < 1e-5, k
    assert out["snapshots"].shape == c["ref32_snapshots"].shape
    assert orc.rel_l2(out["snapshots"], c["ref32_snapshots"]) < 1e-5


@pytest.mark.parametrize("name", CASES)
def test_fp64_gradient_matches_reference_autograd(name):
    c = load_case(name)
    gvp, grho, _ = orc.gradient(**oracle_kwargs(c), res_p=c["lin_p"], res_vx=c["lin_vx"], res_vz=c["lin_vz"],
                                dtype=np.float64)
    assert orc.rel_l2(gvp, c["ref64_grad_vp"]) < 1e-12
    assert orc.rel_l2(grho, c["ref64_grad_rho"]) < 1e-12


def test_layered_100x200_propagator_api():
    c = load_case("layered_100x200")
    out = orc.forward(**oracle_kwargs(c), dtype=np.float64)
    for k in ("p", "vx", "vz"):
        assert orc.rel_l2(out[k], c[f"ref32_{k}"]) < 1e-5, k


def test_fd_coefficients_half_width_4():
    c = orc.fd_coefficients(4)
    np.testing.assert_allclose(c, [1225 / 1024, -245 / 3072, 49 / 5120, -5 / 7168], rtol=1e-13)
    np.testing.assert_allclose(orc.fd_coefficients(2), [9 / 8, -1 / 24], rtol=1e-13)


def test_eighth_order_adjoint_identity():
    """<A w, r> = <w, A^T r> for the 8th-order restatement: the gradient with
    respect to the wavelet (adjoint) dotted with a wavelet perturbation equals
    the trace change (the forward is linear in the wavelet)."""
    c = load_case("small_nofs")
    kw = oracle_kwargs(c)
    kw.update(nt=120, src_v=c["src_v"][:, :120])
    rng = np.random.default_rng(3)
    S, NR = len(c["src_x"]), len(c["rcv_x"])
    res = [rng.standard_normal((S, 120, NR)) for _ in range(3)]
    _, _, gw = orc.gradient(**kw, res_p=res[0], res_vx=res[1], res_vz=res[2], half=4, dtype=np.float64)
    dw = rng.standard_normal((S, 120))
    kw2 = dict(kw, src_v=dw)
    out = orc.forward(**kw2, half=4, dtype=np.float64)
    lhs = sum(float(np.sum(out[k] * r)) for k, r in zip(("p", "vx", "vz"), res))
    rhs = float(np.sum(gw * dw))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_eighth_order_gradient_central_difference():
    """dL/dvp of the 8th-order restatement against central differences."""
    c = load_case("small_nofs")
    kw = oracle_kwargs(c)
    nt = 150
    kw.update(nt=nt, src_v=c["src_v"][:, :nt])
    rng = np.random.default_rng(4)
    S, NR = len(c["src_x"]), len(c["rcv_x"])
    res = rng.standard_normal((S, nt, NR))
    gvp, _, _ = orc.gradient(**kw, res_p=res, half=4, dtype=np.float64)
    dv = rng.standard_normal(c["vp"].shape)
    h = 1e-3
    lp = np.sum(orc.forward(**dict(kw, vp=c["vp"] + h * dv), half=4)["p"] * res)
    lm = np.sum(orc.forward(**dict(kw, vp=c["vp"] - h * dv), half=4)["p"] * res)
    fd = (lp - lm) / (2 * h)
    an = float(np.sum(gvp * dv))
    assert abs(fd - an) <= 1e-6 * abs(an)


def test_row_split_schedule_matches_shot_split():
    """Large grids with fewer shots than threads run the oracle's row loops
    in parallel (the adjoint's scatter loops over alternate row blocks);
    the result must not depend on the thread count.  One thread takes the
    shot loop, the default count splits the rows of this 2-shot grid."""
    nz, nx, nabc, nt = 320, 400, 12, 40
    rng = np.random.default_rng(7)
    vp = (2000 + 800 * rng.random((nz, nx))).astype(np.float64)
    rho = (1800 + 400 * rng.random((nz, nx))).astype(np.float64)
    from geobrain_b200.wave.boundary import bc_pml
    damp = bc_pml(nx, nz, 10.0, 10.0, nabc, float(vp.max()), free_surface=False)
    kw = dict(nz=nz, nx=nx, dz=10.0, nt=nt, dt=1e-3, nabc=nabc, free_surface=True, src_x=np.array([50, 300]),
              src_z=np.array([3, 5]), src_v=rng.standard_normal((2, nt)), rcv_x=np.arange(0, nx, 3),
              rcv_z=np.full(len(range(0, nx, 3)), 2), damp=damp, vp=vp, rho=rho, half=4)
    res = [rng.standard_normal((2, nt, len(kw["rcv_x"]))) for _ in range(3)]
    try:
        orc.set_threads(1)
        f1 = orc.forward(**kw)
        g1 = orc.gradient(**kw, res_p=res[0], res_vx=res[1], res_vz=res[2])
    finally:
        orc.set_threads(0)
    fn = orc.forward(**kw)
    gn = orc.gradient(**kw, res_p=res[0], res_vx=res[1], res_vz=res[2])
    for k in ("p", "vx", "vz", "forward_wavefield_p"):
        assert orc.rel_l2(fn[k], f1[k]) <= 1e-14, k
    for a, b in zip(gn, g1):
        assert orc.rel_l2(a, b) <= 1e-14
