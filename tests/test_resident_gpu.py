"""The resident forward (one launch for many steps, each CTA's tile kept in
shared memory, edge cells sent to the neighbouring tiles as (value, tag)
words through global memory, or stored into their shared memory within a
cluster) against the tile kernel: the same traces and snapshots bit for bit,
the energy maps (summed in another order) to 1e-6; and against the float64
oracle."""
import numpy as np
import pytest

from conftest import load_case, oracle_kwargs
from oracle import oracle as orc
from test_forward_gpu import _plan_of, run_cuda, synthetic_case

pytestmark = pytest.mark.gpu


def _compare(c, device, fd_order, tile_rows=0, snapshot_every=0, mode="global"):
    plan = _plan_of(c, fd_order // 2)
    try:
        plan.set_resident(False)
        base = run_cuda(c, device, fd_order=fd_order, snapshot_every=snapshot_every)
        plan.set_resident(mode, tile_rows)
        info = plan.resident()
        assert info["tile_rows"] > 0
        if tile_rows:
            assert info["tile_rows"] == tile_rows
        out = run_cuda(c, device, fd_order=fd_order, snapshot_every=snapshot_every)
    finally:
        plan.set_resident("auto")
    for k in ("p", "vx", "vz"):
        np.testing.assert_array_equal(out[k], base[k], err_msg=k)
    if snapshot_every:
        np.testing.assert_array_equal(out["snapshots"], base["snapshots"])
    for k in ("forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        assert orc.rel_l2(out[k], base[k]) < 1e-6, k
    return info


@pytest.mark.parametrize("fd_order", [4, 8])
@pytest.mark.parametrize("shape", [(37, 53, 4, 70, 1), (60, 250, 10, 90, 3), (90, 121, 12, 64, 2),
                                   (100, 200, 20, 120, 1)])
def test_resident_matches_tile_kernel(cuda_device, shape, fd_order):
    """Ragged grids, sources and receivers anywhere in the padded grid
    (border cells included), one to three shots."""
    nabc = max(shape[2], fd_order // 2)
    c = synthetic_case(shape[0], shape[1], nabc, shape[3], shape[4], seed=31)
    _compare(c, cuda_device, fd_order)


@pytest.mark.parametrize("tile_rows", [4, 8, 12, 16, 24, 32, 36, 40])
def test_every_tile_height(cuda_device, tile_rows):
    """Every resident tile height, on a grid several tiles tall and wide,
    with snapshots every 16 steps (chunked launches restart from the state
    in global memory)."""
    c = synthetic_case(150, 330, 10, 50, 2, seed=33)
    _compare(c, cuda_device, 8, tile_rows=tile_rows, snapshot_every=16)


# (nabc, tile rows, order): the mirror row fs-1 in the top edge rows of its
# tile, in the bottom edge rows, in the interior rows, and the automatic tiling
FS_CASES = [(12, 8, 8), (9, 12, 8), (12, 16, 8), (12, 0, 4), (12, 0, 8)]


@pytest.mark.parametrize("nabc,tile_rows,fd_order", FS_CASES)
def test_free_surface(cuda_device, nabc, tile_rows, fd_order):
    """Free surface: the mirror rows are set in the tile that owns rows fs-1
    .. fs+1 and sent on after the mirror; sources and receivers at and above
    the surface."""
    c = dict(synthetic_case(70, 260, nabc, 80, 3, seed=35), free_surface=True)
    _compare(c, cuda_device, fd_order, tile_rows=tile_rows, snapshot_every=20)


def test_more_shots_than_one_launch(cuda_device):
    """Forced on with more shots than fit in one cooperative launch: the
    shots run in several launches."""
    c = synthetic_case(300, 900, 20, 40, 4, seed=37)
    info = _compare(c, cuda_device, 8)
    assert info["shots_per_launch"] < 4


@pytest.mark.parametrize("name", ["small_nofs", "small_fs", "layered_100x200"])
def test_resident_matches_reference(cuda_device, name):
    """The automatic choice runs these small single- and few-shot cases
    resident: traces and energies against the reference's own outputs."""
    c = load_case(name)
    plan = _plan_of(c, 2)
    assert plan.resident()["tile_rows"] > 0
    out = run_cuda(c, cuda_device)
    for k in ("p", "vx", "vz", "forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
        assert orc.rel_l2(out[k], c[f"ref32_{k}"]) < 1e-5, k


def test_eighth_order_against_oracle(cuda_device):
    c = synthetic_case(140, 260, 16, 100, 1, seed=39)
    out = run_cuda(c, cuda_device, fd_order=8)
    ref = orc.forward(**oracle_kwargs(dict(c, src_v=c["src_v"])), half=4, dtype=np.float64)
    for k in ("p", "vx", "vz"):
        assert orc.rel_l2(out[k], ref[k]) < 1e-5, k


@pytest.mark.parametrize("fd_order", [4, 8])
@pytest.mark.parametrize("shape,tile_rows", [((37, 53, 4, 70, 1), 0), ((60, 250, 10, 90, 3), 0),
                                             ((90, 121, 12, 64, 2), 0), ((100, 200, 20, 120, 1), 0),
                                             ((150, 330, 10, 50, 2), 36), ((150, 330, 10, 50, 2), 40)])
def test_cluster_exchange_matches_tile_kernel(cuda_device, shape, tile_rows, fd_order):
    """The cluster exchange (one thread-block cluster per shot, halo strips
    read from the neighbours' shared memory, cluster barriers): the tile
    kernel's traces and snapshots bit for bit."""
    nabc = max(shape[2], fd_order // 2)
    c = synthetic_case(shape[0], shape[1], nabc, shape[3], shape[4], seed=43)
    info = _compare(c, cuda_device, fd_order, tile_rows=tile_rows, snapshot_every=16, mode="cluster")
    assert info["exchange"] == "cluster"


@pytest.mark.parametrize("nabc,tile_rows,fd_order", [(12, 8, 8), (9, 12, 8), (12, 0, 4), (12, 0, 8)])
def test_cluster_exchange_free_surface(cuda_device, nabc, tile_rows, fd_order):
    c = dict(synthetic_case(40, 200, nabc, 80, 3, seed=45), free_surface=True)
    info = _compare(c, cuda_device, fd_order, tile_rows=tile_rows, snapshot_every=20, mode="cluster")
    assert info["exchange"] == "cluster"


@pytest.mark.parametrize("shape,tile_rows", [((37, 53, 4, 70, 1), 0), ((60, 250, 10, 90, 3), 0),
                                             ((90, 121, 12, 64, 2), 0), ((100, 200, 20, 120, 1), 0),
                                             ((150, 330, 10, 50, 2), 4), ((150, 330, 10, 50, 2), 8),
                                             ((150, 330, 10, 50, 2), 12), ((150, 330, 10, 50, 2), 16),
                                             ((150, 330, 10, 50, 2), 24), ((150, 330, 10, 50, 2), 40)])
def test_one_exchange_per_step_matches_tile_kernel(cuda_device, shape, tile_rows):
    """4th order without a free surface: p also updated on the neighbours'
    edge rows and columns, v exchanged once a step with all eight
    neighbours; the tile kernel's traces and snapshots bit for bit."""
    c = synthetic_case(shape[0], shape[1], shape[2], shape[3], shape[4], seed=47)
    info = _compare(c, cuda_device, 4, tile_rows=tile_rows, snapshot_every=16, mode="single")
    assert info["exchange"] == "single"


def test_one_exchange_per_step_needs_4th_order_without_free_surface(cuda_device):
    """Asked for only (it measured no faster than two exchanges on 100 x 200);
    refused for the 8th order and with a free surface, and the plan stays
    automatic."""
    from geobrain_b200 import _lib
    c = synthetic_case(100, 200, 20, 30, 1, seed=49)
    assert _plan_of(c, 2).resident()["exchange"] == "global"
    for plan in (_plan_of(c, 4), _plan_of(dict(c, free_surface=True), 2)):
        assert plan._lib.gb_plan_set_resident(plan.h, 3, 0) == _lib.GB_E_UNSUPPORTED
        assert plan.resident()["exchange"] == "global"


def test_invalid_settings(cuda_device):
    """Unknown modes and tile heights are refused; the plan keeps its
    automatic choice."""
    from geobrain_b200 import _lib
    c = synthetic_case(40, 90, 10, 20, 1, seed=41)
    plan = _plan_of(c, 4)
    for mode, rows in ((4, 0), (1, 10), (1, 48), (-2, 0)):
        assert plan._lib.gb_plan_set_resident(plan.h, mode, rows) == _lib.GB_E_ARG
    assert plan.resident()["tile_rows"] > 0
