"""Trajectory sharding over ranks (one process per GPU).

Trajectories are independent (delays of a 2DCS scan, initial states of an adjoint batch, the
lattices of an uneven batch), so the path shards by trajectory with no data-path collective; the
reference scales the same way (MPI split of the delay loop, lattice_md.cpp:929-1500, one GPU per
rank, runners_lattice.cpp:279-284).  Collectives appear only where results meet: the parameter
gradient of a sharded adjoint batch (a sum of <= 5 doubles per trajectory) and the max-over-ranks
timing of the benchmark.

Sums over ranks are formed from an all_gather in rank order, so every rank holds the same,
deterministic result (an all_reduce may order its additions by topology).
"""
from __future__ import annotations

import numpy as np


def scan_delays(n_delays: int, t_max: float, rank: int = 0, world: int = 1) -> np.ndarray:
    """This rank's delays of a world * n_delays point scan of [0, t_max + ...): rank r takes
    t_max * (k + r / world) / (n_delays - 1), k = 0 .. n_delays - 1 (interleaved, equal work)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return t_max * (np.arange(n_delays) + rank / world) / (n_delays - 1)


def shard_lpt(costs, world: int) -> list:
    """Longest-processing-time-first assignment of items with the given costs (e.g. spins x steps
    of each trajectory of an uneven batch) to `world` ranks.  Returns one sorted index list per
    rank; ties go to the lower rank, so every rank computes the same assignment."""
    costs = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(x) for x in out]


def _gather(t, dist):
    import torch
    world = dist.get_world_size()
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    return parts


def sum_over_ranks(values, dist=None, device=None) -> np.ndarray:
    """Sum of a float64 array over ranks, added in rank order (identical on every rank)."""
    import torch
    v = np.ascontiguousarray(values, dtype=np.float64)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return v.copy()
    t = torch.from_numpy(v.copy())
    if device is not None:
        t = t.to(device)
    parts = _gather(t, dist)
    total = parts[0].clone()
    for p in parts[1:]:
        total += p
    return total.cpu().numpy()


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """Largest value of x over ranks (the benchmark times every multi-GPU run this way)."""
    import torch
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sharded_loss_grad(n_traj: int, costs, loss_grad, dist=None):
    """Loss and gradient of a batch of independent trajectories split over ranks.

    ``loss_grad(indices) -> (loss[len], grad[len][n_params])`` evaluates this rank's trajectories
    (on a GPU: ``adjoint.adjoint_rk4`` on their states and targets).  Returns the batch totals
    (sum of losses, sum of gradients), identical on every rank.
    """
    world = dist.get_world_size() if (dist is not None and dist.is_initialized()) else 1
    rank = dist.get_rank() if world > 1 else 0
    mine = shard_lpt(costs if costs is not None else np.ones(n_traj), world)[rank]
    loss, grad = loss_grad(mine)
    grad = np.atleast_2d(np.asarray(grad, dtype=np.float64))
    local = np.concatenate([[float(np.sum(loss))], grad.sum(axis=0) if len(mine) else np.zeros(grad.shape[1])])
    total = sum_over_ranks(local, dist)
    return total[0], total[1:]
