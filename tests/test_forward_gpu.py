"""Forward parity of the CUDA path (through the C ABI) against the reference's
golden outputs and the CPU oracle.  Tolerance: 1e-5 relative L2 in fp32."""
import numpy as np
import pytest
import torch

from conftest import load_case, oracle_kwargs
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-5


def run_cuda(c, device, fd_order=4, **kw):
    from geobrain_b200.wave import acoustic_forward_kernel
    S = len(c["src_x"])
    out = acoustic_forward_kernel(
        nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
        free_surface=c["free_surface"], src_x=torch.as_tensor(c["src_x"]), src_z=torch.as_tensor(c["src_z"]),
        src_n=S, src_v=torch.as_tensor(c["src_v"], device=device), rcv_x=torch.as_tensor(c["rcv_x"]),
        rcv_z=torch.as_tensor(c["rcv_z"]), rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=device),
        vp=torch.as_tensor(c["vp"], device=device), rho=torch.as_tensor(c["rho"], device=device),
        device=device, fd_order=fd_order, **kw)
    torch.cuda.synchronize()
    return {k: (v.cpu().numpy() if torch.is_tensor(v) else v) for k, v in out.items()}


@pytest.mark.parametrize("name", ["small_nofs", "small_fs", "layered_100x200"])
def test_forward_matches_reference(cuda_device, name):
    c = load_case(name)
    out = run_cuda(c, cuda_device)
    for k in ("p", "vx", "vz", "forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        err = orc.rel_l2(out[k], c[f"ref32_{k}"])
        assert err < TOL, (k, err)
        if f"ref64_{k}" in c:
            assert orc.rel_l2(out[k], c[f"ref64_{k}"]) < TOL, k


@pytest.mark.parametrize("name", ["small_nofs", "small_fs"])
def test_snapshots_match_reference(cuda_device, name):
    c = load_case(name)
    out = run_cuda(c, cuda_device, snapshot_every=int(c["snapshot_every"]))
    assert out["snapshots"].shape == c["ref32_snapshots"].shape
    assert orc.rel_l2(out["snapshots"], c["ref32_snapshots"]) < TOL


@pytest.mark.parametrize("free_surface", [False, True])
def test_eighth_order_matches_oracle(cuda_device, free_surface):
    c = load_case("small_fs" if free_surface else "small_nofs")
    ref = orc.forward(**oracle_kwargs(c), half=4, dtype=np.float64)
    out = run_cuda(c, cuda_device, fd_order=8)
    for k in ("p", "vx", "vz", "forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        assert orc.rel_l2(out[k], ref[k]) < TOL, k


def synthetic_case(nz, nx, nabc, nt, n_shots, seed, free_surface=False, edge_rcv=True):
    rng = np.random.default_rng(seed)
    vp = (1800 + 1200 * rng.random((nz, nx))).astype(np.float32)
    rho = (1800 + 400 * rng.random((nz, nx))).astype(np.float32)
    from geobrain_b200.wave import bc_pml, RickerWavelet
    damp = bc_pml(nx, nz, 10.0, 10.0, nabc, float(vp.max()), free_surface=False).astype(np.float32)
    w, _ = RickerWavelet()(f0=20.0, dt=1e-3)
    w = np.pad(w.numpy(), (0, max(0, nt - w.shape[0])))[:nt]
    sx = rng.integers(-nabc, nx + nabc, n_shots)      # sources anywhere in the padded grid, PML included
    sz = rng.integers(-nabc, nz + nabc, n_shots)
    sz[0], sx[0] = -nabc, -nabc                       # a border cell outside every update mask
    rx = np.concatenate([np.arange(0, nx, 3), rng.integers(-nabc, nx + nabc - 1, 40)])
    rz = np.concatenate([np.ones_like(np.arange(0, nx, 3)), rng.integers(-nabc, nz + nabc - 1, 40)])
    if edge_rcv:
        rx = np.concatenate([rx, [-nabc, nx + nabc - 2, 0]])
        rz = np.concatenate([rz, [nz + nabc - 2, -nabc, nz - 1]])
    src_v = (w[None, :] * (1 + rng.random((n_shots, 1)))).astype(np.float32)
    return dict(nz=nz, nx=nx, nabc=nabc, nt=nt, dt=1e-3, dx=10.0, free_surface=free_surface, vp=vp, rho=rho,
                damp=damp, src_x=sx.astype(np.int64), src_z=sz.astype(np.int64), src_v=src_v,
                rcv_x=rx.astype(np.int64), rcv_z=rz.astype(np.int64))


@pytest.mark.parametrize("shape", [(37, 53, 4), (70, 245, 8), (33, 121, 5)])
@pytest.mark.parametrize("fd_order", [4, 8])
def test_ragged_grids_against_oracle(cuda_device, shape, fd_order):
    nz, nx, nabc = shape
    c = synthetic_case(nz, nx, nabc, 90, 3, seed=nz * nx)
    ref = orc.forward(**oracle_kwargs(c), half=fd_order // 2, dtype=np.float64)
    out = run_cuda(c, cuda_device, fd_order=fd_order)
    for k in ("p", "vx", "vz", "forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        assert orc.rel_l2(out[k], ref[k]) < TOL, k


@pytest.mark.parametrize("tiling", [(16, 1), (32, 1), (16, 3), (32, 5), (32, 0)])
def test_tilings_are_bit_identical(cuda_device, tiling):
    """Tile height and shots-per-CTA change the schedule, never the numbers
    (except the energy sums' association order)."""
    c = synthetic_case(90, 250, 10, 60, 7, seed=11)
    plan = _plan_of(c, 4)
    plan.set_resident(False)          # the tile kernel's schedules are what is compared
    try:
        base = run_cuda(c, cuda_device, fd_order=8)
        plan.set_tiling(*tiling)
        out = run_cuda(c, cuda_device, fd_order=8)
    finally:
        plan.set_tiling(32, 0)
        plan.set_resident("auto")
    for k in ("p", "vx", "vz"):
        np.testing.assert_array_equal(out[k], base[k])
    for k in ("forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        assert orc.rel_l2(out[k], base[k]) < 1e-6


def _plan_of(c, half):
    from geobrain_b200.wave import engine
    geo = engine.Geometry(c["nz"], c["nx"], c["nabc"], c["nt"], c["dt"], c["dx"], half, bool(c["free_surface"]))
    return engine.get_plan(geo, c["src_x"], c["src_z"], c["rcv_x"], c["rcv_z"])


@pytest.mark.parametrize("nt,snapshot_every,streams", [(96, 0, True), (101, 32, True), (70, 16, False)])
def test_graph_replay_is_bit_identical(cuda_device, nt, snapshot_every, streams):
    """Chunks of 16 steps replayed from one CUDA graph (step index from a
    device counter; a partial last chunk runs step by step) give the same
    traces and snapshots as one launch per step (the energy sums, added
    with atomics, to their association order); a second call replays the
    cached graph, a call with new buffers captures again."""
    c = synthetic_case(60, 250, 10, nt, 5, seed=3)
    plan = _plan_of(c, 4)
    plan.set_resident(False)               # graphs drive the tile kernel
    plan.set_tiling(16, 2)                 # three groups
    plan.set_group_streams(streams)
    try:
        plan.set_graph_steps(0)
        base = run_cuda(c, cuda_device, fd_order=8, snapshot_every=snapshot_every)
        plan.set_graph_steps(16)
        outs = [run_cuda(c, cuda_device, fd_order=8, snapshot_every=snapshot_every) for _ in range(3)]
    finally:
        plan.set_graph_steps(16)
        plan.set_group_streams(True)
        plan.set_tiling(16, 0)
        plan.set_resident("auto")
    for out in outs:
        for k in ("p", "vx", "vz"):
            np.testing.assert_array_equal(out[k], base[k])
        for k in ("forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
            assert orc.rel_l2(out[k], base[k]) < 1e-6
        if snapshot_every:
            np.testing.assert_array_equal(out["snapshots"], base["snapshots"])


@pytest.mark.parametrize("shape,spc,streams,graph", [
    ((130, 400, 20, 40, 7), 2, True, 16),    # every item split (fewer items than resident CTAs); a 1-shot group
    ((130, 400, 20, 40, 7), 2, False, 0),    # one launch for all groups, step by step
    ((400, 1200, 30, 12, 32), 0, True, 16),  # the 400 x 1200, 32-shot workload: only the last items split
])
def test_cta_schedule_does_not_change_results(cuda_device, shape, spc, streams, graph):
    """The guided CTA order (slow-path tiles first, the forward's last
    items split into halves of their shots) against blockIdx order: traces
    and snapshots bit for bit, energies (atomic sums) to 1e-6.  A missing
    item would leave stale cells, a doubled one doubled energies."""
    c = synthetic_case(*shape, seed=41)
    plan = _plan_of(c, 4)
    plan.set_resident(False)
    plan.set_tiling(16, spc)
    plan.set_group_streams(streams)
    plan.set_graph_steps(graph)
    try:
        plan.set_schedule(0)
        base = run_cuda(c, cuda_device, fd_order=8, snapshot_every=4)
        plan.set_schedule(1)
        out = run_cuda(c, cuda_device, fd_order=8, snapshot_every=4)
    finally:
        plan.set_schedule(0)
        plan.set_graph_steps(16)
        plan.set_group_streams(True)
        plan.set_tiling(16, 0)
        plan.set_resident("auto")
    for k in ("p", "vx", "vz"):
        np.testing.assert_array_equal(out[k], base[k], err_msg=k)
    np.testing.assert_array_equal(out["snapshots"], base["snapshots"])
    for k in ("forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        assert orc.rel_l2(out[k], base[k]) < 1e-6, k
    assert np.abs(out["p"]).max() > 0


def test_graph_steps_validation(cuda_device):
    c = synthetic_case(40, 130, 10, 20, 1, seed=2)
    plan = _plan_of(c, 4)
    for bad in (3, -2, 66):
        with pytest.raises(Exception):
            plan.set_graph_steps(bad)


def test_autotune_picks_a_configuration_and_keeps_results(cuda_device):
    """The autotuner only changes the launch configuration: traces after
    tuning equal those before."""
    c = synthetic_case(80, 300, 10, 48, 6, seed=9)
    base = run_cuda(c, cuda_device, fd_order=8)
    plan = _plan_of(c, 4)
    assert plan.tuned is None
    try:
        tuned = run_cuda(c, cuda_device, fd_order=8, autotune=True)
        cfg = plan.tuned
        assert cfg is not None and cfg["ms_per_step"] > 0
        assert cfg["tile_rows"] in (16, 32) and cfg["graph_steps"] in (0, 16)
        assert plan.config() == {k: cfg[k] for k in ("tile_rows", "shots_per_cta", "group_streams", "graph_steps",
                                                     "stream_chunks", "resident_rows")}
    finally:
        plan.set_graph_steps(16)
        plan.set_streaming(False)
        plan.set_group_streams(True)
        plan.set_tiling(16, 0)
        plan.set_resident("auto")
    for k in ("p", "vx", "vz"):
        np.testing.assert_array_equal(tuned[k], base[k])


def test_wavelet_scaling_is_linear(cuda_device):
    """Linearity in the source at a large grid (a size-independent check):
    doubling the wavelet doubles every trace to fp32 rounding.  Bit-exact
    doubling does not hold for this scheme in fp32 even on the CPU oracle
    (about one sample in thirty moves by one ulp), so the bar is the
    rounding level, 1e-6 relative L2."""
    c = synthetic_case(300, 900, 20, 200, 4, seed=5)
    a = run_cuda(c, cuda_device, fd_order=8)
    c2 = dict(c, src_v=c["src_v"] * 2)
    b = run_cuda(c2, cuda_device, fd_order=8)
    for k in ("p", "vx", "vz"):
        assert np.abs(a[k]).max() > 0
        assert orc.rel_l2(b[k], 2 * a[k]) < 1e-6, k


def test_shots_are_independent(cuda_device):
    """Each shot's traces do not depend on which other shots share the launch."""
    c = synthetic_case(120, 300, 12, 80, 5, seed=9)
    allr = run_cuda(c, cuda_device)
    for s in (0, 3):
        one = dict(c, src_x=c["src_x"][s:s + 1], src_z=c["src_z"][s:s + 1], src_v=c["src_v"][s:s + 1])
        o = run_cuda(one, cuda_device)
        for k in ("p", "vx", "vz"):
            np.testing.assert_array_equal(o[k][0], allr[k][s])


def test_invalid_positions_raise(cuda_device):
    c = synthetic_case(40, 60, 5, 10, 2, seed=1)
    bad = dict(c, rcv_x=np.array([c["nx"] + c["nabc"] - 1]), rcv_z=np.array([0]))
    with pytest.raises(ValueError):
        run_cuda(bad, cuda_device)
    bad = dict(c, src_x=np.array([0, -c["nabc"] - 1]))
    with pytest.raises(ValueError):
        run_cuda(bad, cuda_device)


def test_cpu_device_is_rejected():
    from geobrain_b200.wave import acoustic_forward_kernel
    c = load_case("small_nofs")
    with pytest.raises(ValueError):
        acoustic_forward_kernel(nx=c["nx"], nz=c["nz"], dx=10.0, dz=10.0, nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
                                free_surface=False, src_x=c["src_x"], src_z=c["src_z"], src_n=3,
                                src_v=torch.as_tensor(c["src_v"]), rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
                                rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"]),
                                vp=torch.as_tensor(c["vp"]), rho=torch.as_tensor(c["rho"]),
                                device=torch.device("cpu"))


@pytest.mark.parametrize("shape,chunks,order", [((60, 250, 10, 70, 5), 0, 8), ((90, 121, 12, 50, 3), 1, 8),
                                                 ((45, 250, 8, 60, 2), 2, 8), ((300, 900, 20, 40, 4), 3, 8),
                                                 ((70, 200, 10, 60, 3), 2, 4)])
def test_streaming_kernel_is_bit_identical(cuda_device, shape, chunks, order):
    """The streaming forward kernel (each CTA walks a column strip of one
    shot down a z-segment) gives the tile kernel's traces and snapshots bit
    for bit, on ragged grids with sources and receivers on the padded border
    and for every segment length (the energy sums, added in another order,
    to 1e-6)."""
    c = synthetic_case(*shape, seed=21)
    plan = _plan_of(c, order // 2)
    plan.set_tiling(16, 0)
    plan.set_resident(False)
    try:
        base = run_cuda(c, cuda_device, fd_order=order, snapshot_every=16)
        plan.set_streaming(True, chunks)
        assert plan.config()["stream_chunks"] > 0
        out = run_cuda(c, cuda_device, fd_order=order, snapshot_every=16)
    finally:
        plan.set_streaming(False)
        plan.set_resident("auto")
    for k in ("p", "vx", "vz"):
        np.testing.assert_array_equal(out[k], base[k])
    np.testing.assert_array_equal(out["snapshots"], base["snapshots"])
    for k in ("forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        assert orc.rel_l2(out[k], base[k]) < 1e-6


def test_streaming_kernel_is_not_used_with_a_free_surface(cuda_device):
    c = dict(synthetic_case(60, 250, 10, 30, 2, seed=4), free_surface=True)
    plan = _plan_of(c, 4)
    plan.set_resident(False)
    plan.set_streaming(True, 0)
    try:
        assert plan.config()["stream_chunks"] == 0          # the tile kernel runs
        out = run_cuda(c, cuda_device, fd_order=8)
        plan.set_streaming(False)
        base = run_cuda(c, cuda_device, fd_order=8)
    finally:
        plan.set_streaming(False)
        plan.set_resident("auto")
    np.testing.assert_array_equal(out["p"], base["p"])


@pytest.mark.parametrize("nabc,tile_rows,resident", [(12, 16, False), (16, 16, False), (16, 32, False),
                                                     (12, 0, True)])
def test_receivers_above_the_free_surface(cuda_device, nabc, tile_rows, resident):
    """Receivers in row fs-1 (one above the surface) record vz after the
    mirror vz[fs-1] = vz[fs] of the same step (acoustic_2d.py:268-274): the
    tile kernel takes their vz from the tile that updates row fs (the same
    tile, or, with nabc = 16 and 16-row tiles, the next one).  Every
    receiver's traces against the float64 oracle; receivers in rows fs-1,
    fs and fs+1."""
    c = dict(synthetic_case(50, 200, nabc, 150, 2, seed=7), free_surface=True)
    rx = np.arange(0, 200, 7)
    c["rcv_x"] = np.concatenate([rx, rx, rx])
    c["rcv_z"] = np.concatenate([np.full(rx.size, -1), np.zeros(rx.size, np.int64), np.ones(rx.size, np.int64)])
    c["src_z"] = np.array([0, 3])
    c["src_x"] = np.array([40, 150])
    plan = _plan_of(c, 4)
    plan.set_resident(resident)
    if tile_rows:
        plan.set_tiling(tile_rows, 0)
    try:
        out = run_cuda(c, cuda_device, fd_order=8)
        if resident:
            assert plan.resident()["tile_rows"] > 0
    finally:
        plan.set_tiling(0, 0)
        plan.set_resident("auto")
    ref = orc.forward(**oracle_kwargs(c), half=4, dtype=np.float64)
    for k in ("p", "vx", "vz"):
        # per receiver, relative to its own trace (or to a thousandth of the
        # field's, for traces the wave has barely reached)
        floor = 1e-3 * np.linalg.norm(ref[k]) / np.sqrt(c["rcv_x"].size)
        for r in range(c["rcv_x"].size):
            err = np.linalg.norm(out[k][:, :, r] - ref[k][:, :, r]) / max(np.linalg.norm(ref[k][:, :, r]), floor)
            assert err < TOL, (k, r, c["rcv_z"][r], err)
