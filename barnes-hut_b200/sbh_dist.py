"""Multi-GPU host logic. The summation path shards without any data-path
collective: a forest of independent systems is split by system across ranks
(each rank builds and evaluates its own systems), and a single large system
runs as independent replicas. The only collectives are for timing and
bookkeeping: a barrier, the max of the per-rank step times, and gathering
per-rank counts. Process groups come from torch.distributed (nccl on GPUs,
gloo on CPU)."""
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
