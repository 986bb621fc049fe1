"""Multi-GPU host logic. Two ways to spread the summation over ranks:

* by system, with no data-path collective: a forest of independent systems
  is split by system across ranks (each rank builds and evaluates its own
  systems), and a single system can run as independent replicas;
* by target, for one large system: every rank builds the same tree and walks
  the target groups of its share of the sorted positions
  (sbh_native_set_target_range), then one all-reduce (sum) of the forces and
  of the position and mass gradients (N x 28 bytes) gives every rank the
  full result. Queries are independent given the sources, and the
  source-side adjoint is a sum over targets, so the sum over ranks is exact
  up to FP32 summation order.

Other collectives are for timing and bookkeeping: a barrier, the max of the
per-rank step times, and gathering per-rank counts. Process groups come from
torch.distributed (nccl on GPUs, gloo on CPU)."""
from __future__ import annotations

import numpy as np


def shard_systems(sizes, world: int, rank: int):
    """Contiguous block of system indices for `rank`, balancing the particle
    count (greedy split of the prefix sums). Returns (first, last+1)."""
    sizes = np.asarray(sizes, dtype=np.int64)
    if world <= 1 or sizes.size == 0:
        return 0, int(sizes.size)
    cum = np.concatenate([[0], np.cumsum(sizes)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(cum, target, side="left"))
        if b > 0 and abs(cum[b - 1] - target) <= abs(cum[min(b, sizes.size)] - target):
            b -= 1
        bounds.append(b)
    bounds.append(int(sizes.size))
    bounds = np.maximum.accumulate(np.asarray(bounds))
    return int(bounds[rank]), int(bounds[rank + 1])


def system_offsets(sizes) -> np.ndarray:
    """int64 offsets (num_systems + 1) of systems concatenated in order."""
    return np.concatenate([[0], np.cumsum(np.asarray(sizes, dtype=np.int64))]).astype(np.int64)


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (a step time) over the default process group;
    identity without one."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def shard_targets(n: int, world: int, rank: int):
    """[begin, end) of the sorted target positions rank `rank` serves: equal
    shares of [0, n), contiguous and in rank order, so the ranks partition
    the targets."""
    if world <= 1:
        return 0, int(n)
    return int(n * rank // world), int(n * (rank + 1) // world)


def _all_reduce_sum(tensors):
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return
    for t in tensors:
        if t is not None:
            dist.all_reduce(t, op=dist.ReduceOp.SUM)


def sharded_force(tree, **params):
    """Force of one system with its targets split across the ranks of the
    default process group: each rank walks its share of the target groups of
    the same tree, then the force rows (zero outside each rank's share) are
    summed over ranks. Returns the full (N, 3) force on every rank."""
    import torch.distributed as dist

    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    b, e = shard_targets(tree.n, world, rank)
    tree.set_target_range(b, e)
    try:
        f = tree.force(**params)
    finally:
        tree.set_target_range(0, tree.n)
    _all_reduce_sum([f])
    return f


def sharded_force_vjp(tree, cotangent, *, want_force: bool = True, **params):
    """(force or None, d/d points, d/d masses) of sum(cotangent * force) for
    one system with its targets split across ranks: each rank's walk covers
    its share of the target groups, its finalize spreads the node adjoints it
    collected to every particle, and the sum over ranks of forces and
    gradients is the full result, on every rank."""
    import torch.distributed as dist

    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    b, e = shard_targets(tree.n, world, rank)
    tree.set_target_range(b, e)
    try:
        f, gx, gm = tree.force_vjp(cotangent, want_force=want_force, **params)
    finally:
        tree.set_target_range(0, tree.n)
    _all_reduce_sum([f, gx, gm])
    return f, gx, gm
