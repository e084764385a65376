"""Multi-rank host logic on CPU: world_size-2 gloo process groups.

The path shards by trajectory with no data-path collective; these tests check the assignment
(complete, disjoint, identical on every rank, balanced), the deterministic rank-ordered sums and
max-over-ranks timing, and a sharded adjoint batch whose per-trajectory gradients come from the
oracle's FP64 tangent-linear model (the GPU path passes adjoint.adjoint_rk4 instead).
"""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from classical_mcmc_spin_b200 import sharding
        res = {}
        costs = np.array([128, 3456, 512, 8192, 1152, 2048, 1024, 288, 8192, 4608]) * 1000.0
        res["lpt"] = sharding.shard_lpt(costs, world)
        res["delays"] = sharding.scan_delays(256, 100.0, rank, world)
        res["sum"] = sharding.sum_over_ranks(np.array([rank + 0.1, 2.0 * rank, 1e-17]), dist)
        res["max"] = sharding.max_over_ranks(10.0 + rank, dist)

        import ll_oracle
        L = ll_oracle.OracleLattice.kitaev(3, 3, 1, h=0.1, direction=(0, 1, 0), K=-1.0, Gamma=0.25, Gammap=-0.02)
        basis = [ll_oracle.OracleLattice.kitaev(3, 3, 1, h=e[4], direction=(0, 1, 0), K=e[0], Gamma=e[1],
                                                Gammap=e[2], J=e[3]) for e in np.eye(5)]
        from classical_mcmc_spin_b200.states import random_unit_spins
        S, dt, B = 20, 0.01, 5
        states = [random_unit_spins(L.N, 300 + b).ravel() for b in range(B)]
        targets = [np.random.default_rng(b).normal(scale=0.05, size=(S + 1, 3)) for b in range(B)]

        def loss_grad(idx):
            ls, gs = [], []
            for b in idx:
                l, g = ll_oracle.loss_grad_tlm(L, basis, states[b], 0.0, dt, S, targets[b])
                ls.append(l)
                gs.append(g)
            return np.array(ls), np.array(gs).reshape(len(idx), 5)

        res["adj"] = sharding.sharded_loss_grad(B, np.ones(B), loss_grad, dist)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.array(res, dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_with_gloo(tmp_path, oracle):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    r = [np.load(tmp_path / f"rank{k}.npy", allow_pickle=True).item() for k in range(world)]
    # identical assignment on both ranks, complete and disjoint, balanced within one item
    assert r[0]["lpt"] == r[1]["lpt"]
    parts = r[0]["lpt"]
    assert sorted(parts[0] + parts[1]) == list(range(10))
    costs = np.array([128, 3456, 512, 8192, 1152, 2048, 1024, 288, 8192, 4608]) * 1000.0
    loads = [costs[p].sum() for p in parts]
    assert abs(loads[0] - loads[1]) <= costs.max()
    # the two ranks' delays interleave into one 512-point scan without overlap
    d = np.sort(np.concatenate([r[0]["delays"], r[1]["delays"]]))
    assert len(np.unique(d)) == 512 and d[0] == 0.0
    # sums in rank order, identical on every rank; max over ranks
    for k in range(world):
        np.testing.assert_array_equal(r[k]["sum"], np.array([0.1, 0.0, 1e-17]) + np.array([1.1, 2.0, 1e-17]))
        assert r[k]["max"] == 11.0
    # sharded adjoint batch == serial sum of the per-trajectory tangent-linear gradients
    L = oracle.OracleLattice.kitaev(3, 3, 1, h=0.1, direction=(0, 1, 0), K=-1.0, Gamma=0.25, Gammap=-0.02)
    basis = [oracle.OracleLattice.kitaev(3, 3, 1, h=e[4], direction=(0, 1, 0), K=e[0], Gamma=e[1], Gammap=e[2],
                                         J=e[3]) for e in np.eye(5)]
    from classical_mcmc_spin_b200.states import random_unit_spins
    lt, gt = 0.0, np.zeros(5)
    for b in range(5):
        l, g = oracle.loss_grad_tlm(L, basis, random_unit_spins(L.N, 300 + b).ravel(), 0.0, 0.01, 20,
                                    np.random.default_rng(b).normal(scale=0.05, size=(21, 3)))
        lt += l
        gt += g
    for k in range(world):
        loss, grad = r[k]["adj"]
        assert abs(loss - lt) <= 1e-12 * abs(lt)
        np.testing.assert_allclose(grad, gt, rtol=1e-12, atol=1e-15)


def test_single_rank_fallbacks():
    from classical_mcmc_spin_b200 import sharding
    assert sharding.shard_lpt([3.0, 1.0, 2.0], 1) == [[0, 1, 2]]
    np.testing.assert_array_equal(sharding.sum_over_ranks([1.0, 2.0]), [1.0, 2.0])
    assert sharding.max_over_ranks(3.5) == 3.5
    np.testing.assert_allclose(sharding.scan_delays(256, 100.0), 100.0 * np.arange(256) / 255.0)
    with pytest.raises(ValueError):
        sharding.scan_delays(4, 1.0, 2, 2)
