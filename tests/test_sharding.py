"""Multi-rank host logic of the sharded paths (geobrain_b200.wave.sharding),
run as world_size-2 gloo process groups on the CPU.  The rank-local compute
is the float64 CPU oracle (shot gradient) or a small linear forward model
(ensemble log-likelihood), so what is tested is the split, the empty-rank
case and the single packed all-reduce: the two-rank totals must equal the
one-process totals."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_case, oracle_kwargs
from geobrain_b200.wave import sharding


def test_partition_covers_disjoint_and_balances():
    w = [5, 1, 1, 1, 3, 3, 2, 8]
    parts = [sharding.partition(w, 3, r) for r in range(3)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(w)))
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(w)
    assert all(p == sorted(p) for p in parts)
    assert sharding.partition([1, 1, 1], 4, 3) == []          # more ranks than items
    with pytest.raises(ValueError):
        sharding.partition([1], 2, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_local_fn(c, d_obs):
    from oracle import oracle as orc
    kw = oracle_kwargs(c)

    def run(shots):
        if not shots:
            return torch.zeros((), dtype=torch.float64), torch.zeros(c["vp"].shape, dtype=torch.float64)
        sub = dict(kw, src_x=kw["src_x"][shots], src_z=kw["src_z"][shots], src_v=kw["src_v"][shots])
        pred = orc.forward(**sub, half=4, dtype=np.float64)["p"]
        r = pred - d_obs[shots]
        gvp, _, _ = orc.gradient(**sub, res_p=r, half=4, dtype=np.float64)
        return torch.tensor(0.5 * float((r * r).sum()), dtype=torch.float64), torch.from_numpy(np.asarray(gvp))

    return run


def _shot_worker(rank, world, port, out_dir, n_shots):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = load_case("small_nofs")
        d_obs = (c["ref32_p"] * 0.9).astype(np.float64)
        keep = list(range(n_shots))
        c = dict(c, src_x=c["src_x"][keep], src_z=c["src_z"][keep], src_v=c["src_v"][keep])
        loss, grad = sharding.sharded_shot_gradient(n_shots, _oracle_local_fn(c, d_obs[keep]))
        torch.save({"loss": loss, "grad": grad}, os.path.join(out_dir, f"shot{rank}.pt"))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_shots", [3, 1])
def test_two_rank_shot_gradient_matches_one_process(tmp_path, n_shots):
    """3 shots: ranks take 2 and 1; 1 shot: rank 1 has nothing and adds zeros."""
    mp.spawn(_shot_worker, args=(2, _free_port(), str(tmp_path), n_shots), nprocs=2, join=True)
    c = load_case("small_nofs")
    keep = list(range(n_shots))
    c = dict(c, src_x=c["src_x"][keep], src_z=c["src_z"][keep], src_v=c["src_v"][keep])
    d_obs = (load_case("small_nofs")["ref32_p"] * 0.9).astype(np.float64)[keep]
    loss1, grad1 = _oracle_local_fn(c, d_obs)(keep)
    for r in range(2):
        got = torch.load(os.path.join(tmp_path, f"shot{r}.pt"))
        np.testing.assert_allclose(float(got["loss"]), float(loss1), rtol=1e-12)
        np.testing.assert_allclose(got["grad"].numpy(), grad1.numpy(), rtol=1e-10, atol=1e-12 * float(
            np.abs(grad1.numpy()).max()))


def _linear_problem():
    g = torch.Generator().manual_seed(0)
    A = torch.randn(6, 9, generator=g, dtype=torch.float64)
    obs = torch.randn(9, generator=g, dtype=torch.float64)
    theta = torch.randn(5, 6, generator=g, dtype=torch.float64)
    return A, obs, theta


def _ll_worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A, obs, theta = _linear_problem()
        ll, grad = sharding.sharded_log_likelihood(theta, lambda th: th @ A, obs, noise_std=0.5,
                                                   weights=[1, 2, 3, 4, 5])
        torch.save({"ll": ll, "grad": grad}, os.path.join(out_dir, f"ll{rank}.pt"))
    finally:
        dist.destroy_process_group()


def test_two_rank_log_likelihood_matches_per_particle_loop(tmp_path):
    mp.spawn(_ll_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    A, obs, theta = _linear_problem()
    # the reference's loop (geobrain/core/inverse.py:104-110), one particle at a time
    lls, grads = [], []
    for i in range(theta.shape[0]):
        t = theta[i].clone().requires_grad_(True)
        r = (t @ A - obs) / 0.5
        ll = -0.5 * (r * r).sum()
        ll.backward()
        lls.append(float(ll.detach()))
        grads.append(t.grad.clone())
    for rank in range(2):
        got = torch.load(os.path.join(tmp_path, f"ll{rank}.pt"))
        np.testing.assert_allclose(got["ll"].numpy(), np.array(lls), rtol=1e-13)
        np.testing.assert_allclose(got["grad"].numpy(), torch.stack(grads).numpy(), rtol=1e-12)


def test_single_process_needs_no_process_group():
    A, obs, theta = _linear_problem()
    ll, grad = sharding.sharded_log_likelihood(theta, lambda th: th @ A, obs, with_grad=False)
    assert grad is None and ll.shape == (5,)
    loss, g = sharding.sharded_shot_gradient(2, lambda s: (torch.tensor(float(len(s))), torch.ones(3) * len(s)))
    assert float(loss) == 2.0 and torch.equal(g, torch.full((3,), 2.0))
