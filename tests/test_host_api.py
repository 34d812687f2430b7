"""Host-side mirror of the reference API (CPU only): boundary profile, padding,
wavelet, configuration validation, survey, model, result container, and the
synthetic workload generators."""
import numpy as np
import pytest
import torch

from conftest import load_case
from geobrain_b200 import synthetic, wave


@pytest.mark.parametrize("name", ["small_nofs", "small_fs", "layered_100x200"])
def test_bc_pml_matches_reference(name):
    c = load_case(name)
    damp = wave.bc_pml(c["nx"], c["nz"], c["dx"], c["dx"], c["nabc"], float(c["vp"].max()), free_surface=False)
    np.testing.assert_allclose(damp.astype(np.float32), c["damp"], rtol=1e-6, atol=0)


def test_bc_pml_free_surface_shape_and_top():
    d = wave.bc_pml(50, 30, 10.0, 10.0, 8, 3000.0, free_surface=True)
    assert d.shape == (30 + 8, 50 + 16)
    assert np.all(d[0, 8:-8] == 0)          # no top layer
    assert d[-1, 20] > 0 and d[10, 0] > 0


def test_create_boundary_errors():
    with pytest.raises(ValueError):
        wave.create_boundary("pml", 10, 10, 1.0, 1.0, 4)            # vmax missing
    with pytest.raises(ValueError):
        wave.create_boundary("nope", 10, 10, 1.0, 1.0, 4, vmax=1.0)
    with pytest.raises(NotImplementedError):
        wave.create_boundary("gerjan", 10, 10, 1.0, 1.0, 4)
    with pytest.raises(ZeroDivisionError):
        wave.bc_pml(10, 10, 1.0, 1.0, 1, 1000.0)


def test_pad_model_matches_reference():
    c = load_case("small_nofs")
    out = wave.pad_model(torch.tensor(c["vp"]), c["nabc"], c["nz"], c["nx"])
    np.testing.assert_array_equal(out.numpy(), c["pad_vp"])


def test_ricker_matches_reference():
    c = load_case("layered_100x200")
    w, t = wave.RickerWavelet()(f0=c["f0"], dt=c["dt"])
    n = w.shape[0]
    np.testing.assert_allclose(w.numpy(), c["wavelet"][:n], rtol=1e-6, atol=1e-7)
    assert np.all(c["wavelet"][n:] == 0)
    np.testing.assert_allclose(synthetic.ricker(c["f0"], c["dt"], c["nt"]), c["wavelet"], rtol=1e-5, atol=1e-6)
    w2, t2 = wave.create_wavelet("ricker", f0=c["f0"], dt=c["dt"], nt=c["nt"])
    assert w2.shape[0] == c["nt"] and t2.shape[0] == c["nt"]


def test_config_validation():
    with pytest.raises(ValueError):
        wave.GridConfig(nx=10, nz=10, dx=10.0, dz=5.0)
    with pytest.raises(ValueError):
        wave.GridConfig(nx=0, nz=10, dx=10.0, dz=10.0)
    with pytest.raises(ValueError):
        wave.BoundaryConfig(type="abc")
    with pytest.raises(ValueError):
        wave.BoundaryConfig(n_layers=0)
    with pytest.raises(ValueError):
        wave.SolverConfig(fd_order=5)
    with pytest.raises(ValueError):
        wave.TimeConfig(nt=0, dt=1.0)
    g = wave.GridConfig(nx=200, nz=100, dx=10.0, dz=10.0)
    assert g.shape == (100, 200) and g.ndim == 2 and g.extent == (0.0, 1990.0, 990.0, 0.0)
    assert wave.WaveletConfig(f0=25.0).delay == pytest.approx(0.048)


def test_survey_and_model():
    nt, dt = 100, 1e-3
    src = wave.Source(nt=nt, dt=dt, f0=10.0)
    src.add_sources(np.arange(2, 20, 5), np.ones(4, int), np.ones(nt))
    src.add_source(3, 4, np.ones(nt))
    assert src.num == 5 and src.get_loc().shape == (5, 2) and src.get_wavelet().shape == (5, nt)
    with pytest.raises(ValueError):
        src.add_source(1, 1, np.ones(nt - 1))
    rcv = wave.Receiver(nt=nt, dt=dt)
    rcv.add_receivers(np.arange(10), np.ones(10, int), "pr")
    with pytest.raises(ValueError):
        rcv.add_receiver(1, 1, "xx")
    sv = wave.Survey(src, rcv)
    assert (sv.n_shots, sv.n_receivers, sv.nt, sv.dt, sv.f0) == (5, 10, nt, dt, 10.0)
    with pytest.raises(ValueError):
        sv.set_receiver_masks(np.ones((2, 2)))
    grid = wave.GridConfig(nx=20, nz=10, dx=10.0, dz=10.0)
    vp = np.full((10, 20), 2500.0, np.float32)
    m = wave.AcousticModel(grid, wave.BoundaryConfig(n_layers=5), vp=vp, rho=np.ones_like(vp),
                           vp_bound=(2000.0, 2400.0), vp_grad=True)
    m.forward()
    # Gardner's density comes from vp before clipping (models/acoustic.py:190-195)
    np.testing.assert_allclose(m.rho.detach().numpy(), 310.0 * 2500.0 ** 0.25, rtol=1e-6)
    assert float(m.vp.detach().max()) == 2400.0
    with pytest.raises(ValueError):
        wave.AcousticModel(grid, wave.BoundaryConfig(), vp=vp[:5], rho=vp[:5])
    r = wave.WaveResult(p=torch.zeros(1, 2, 3), vx=torch.zeros(1), vz=torch.zeros(1),
                        forward_wavefield_p=torch.zeros(1), forward_wavefield_vx=torch.zeros(1),
                        forward_wavefield_vz=torch.zeros(1))
    assert r["p"].shape == (1, 2, 3) and "snapshots" not in r and r.n_receivers == 3
    with pytest.raises(KeyError):
        r["nope"]


def test_propagator_rejects_cpu_forward():
    grid = wave.GridConfig(nx=20, nz=10, dx=10.0, dz=10.0)
    vp = np.full((10, 20), 2500.0, np.float32)
    m = wave.AcousticModel(grid, wave.BoundaryConfig(n_layers=5), vp=vp, rho=np.ones_like(vp) * 2000,
                           auto_update_rho=False)
    src = wave.Source(nt=10, dt=1e-3, f0=10.0)
    src.add_source(5, 1, np.ones(10))
    rcv = wave.Receiver(nt=10, dt=1e-3)
    rcv.add_receivers(np.arange(20), np.ones(20, int), "pr")
    prop = wave.AcousticPropagator(m, wave.Survey(src, rcv), device="cpu")
    assert prop.damp.shape == (20, 30)
    with pytest.raises(ValueError):
        prop.forward()


def test_synthetic_workloads_are_seeded_and_stable():
    a = synthetic.gaussian_field(64, 128, 10.0, 50.0, 200.0, seed=3)
    b = synthetic.gaussian_field(64, 128, 10.0, 50.0, 200.0, seed=3)
    np.testing.assert_array_equal(a, b)
    assert abs(a.std() - 1.0) < 1e-9 and abs(a.mean()) < 1e-9
    # anisotropy: correlation decays slower along x than along z
    cx = np.mean(a[:, :-5] * a[:, 5:])
    cz = np.mean(a[:-5, :] * a[5:, :])
    assert cx > cz
    w1 = synthetic.plain_forward_100x200()
    assert w1.vp.shape == (100, 200) and w1.n_shots == 1 and w1.fd_order == 4
    assert synthetic.cfl_number(float(w1.vp.max()), w1.dt, w1.dx, 4) < 1.0


def test_fwi_workload_shape_and_cfl():
    w = synthetic.fwi_400x1200(nt=10)
    assert w.vp.shape == (400, 1200) and w.n_shots == 32 and w.rcv_x.size == 1200
    assert w.cells == 460 * 1260
    assert synthetic.cfl_number(float(w.vp_true.max()), w.dt, w.dx, 8) < 1.0
    assert np.abs(w.vp - w.vp_true).mean() > 1.0          # initial model is smoothed


def test_uneven_batch_covers_sizes():
    ms = synthetic.uneven_batch(24, nt_scale=0.01)
    assert len(ms) == 24
    assert all(4 <= m.n_shots <= 16 for m in ms)
    assert all(m.vp.min() >= 1500 and m.vp.max() <= 4500 for m in ms)


def test_courant_number_and_input_checks():
    """The host checks the boundary runs before a launch: the Courant number
    of the staggered scheme (stable below 1), finite and positive models and
    finite wavelets."""
    import torch
    from geobrain_b200.wave import engine
    # 4th order, 2-D: vmax dt / dx * (9/8 + 1/24) * sqrt(2)
    assert abs(engine.courant_number(3000.0, 1e-3, 10.0, 4) - 0.3 * (7 / 6) * 2 ** 0.5) < 1e-12
    assert engine.courant_number(3000.0, 1e-3, 10.0, 8) > engine.courant_number(3000.0, 1e-3, 10.0, 4)
    assert abs(engine.courant_number(1.0, 1.0, 1.0, 4, ndim=3) / engine.courant_number(1.0, 1.0, 1.0, 4) -
               (3 / 2) ** 0.5) < 1e-12
    vp = torch.full((8, 9), 3000.0)
    rho = torch.full((8, 9), 2000.0)
    w = torch.zeros(2, 5)
    assert engine.check_model_inputs(vp, rho, w, 1e-3, 10.0, 8) == 3000.0
    with pytest.raises(ValueError, match="Courant"):
        engine.check_model_inputs(vp, rho, w, 3e-3, 10.0, 8)
    with pytest.raises(ValueError, match="Courant"):
        engine.check_model_inputs(vp, rho, w, 2e-3, 10.0, 4, ndim=3)
    bad = vp.clone()
    bad[3, 4] = float("nan")
    with pytest.raises(ValueError, match="vp has non-finite"):
        engine.check_model_inputs(bad, rho, w, 1e-3, 10.0, 8)
    with pytest.raises(ValueError, match="rho must be positive"):
        engine.check_model_inputs(vp, -rho, w, 1e-3, 10.0, 8)
    with pytest.raises(ValueError, match="src_v has non-finite"):
        engine.check_model_inputs(vp, rho, w + float("inf"), 1e-3, 10.0, 8)


def test_plan_sub_batches():
    """Consecutive sub-batches of the fused batched gradient, by memory."""
    from geobrain_b200.wave.batched import plan_sub_batches
    assert plan_sub_batches([3, 3, 3, 3], 7) == [[0, 1], [2, 3]]
    assert plan_sub_batches([5, 9, 1], 6) == [[0], [1], [2]]
    assert plan_sub_batches([1, 1, 1], 100) == [[0, 1, 2]]
    # as few as a greedy fill, but even: not [5 models] + [1]
    assert plan_sub_batches([2] * 6, 10) == [[0, 1, 2], [3, 4, 5]]
    groups = plan_sub_batches([4, 1, 3, 2, 5, 1, 2, 3], 11)
    assert len(groups) == 2 and sorted(i for g in groups for i in g) == list(range(8))
    assert max(sum([4, 1, 3, 2, 5, 1, 2, 3][i] for i in g) for g in groups) <= 11
    assert [len(g) for g in plan_sub_batches([3] * 10, 20)] == [5, 5]
