"""World-size-2 gloo tests (CPU) of the multi-GPU host logic: forest
sharding by system covers every system exactly once with balanced particle
counts, and the step time reported is the max over ranks."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import sbh_dist


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    a, b = sbh_dist.shard_systems(sizes, world, rank)
    mine = float(sum(sizes[a:b]))
    total = sbh_dist.sum_over_ranks(mine)
    slowest = sbh_dist.max_over_ranks(10.0 + rank)
    out[rank] = (a, b, total, slowest)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_and_timing():
    rng = np.random.default_rng(0)
    sizes = list(np.exp(rng.uniform(np.log(1000), np.log(200000), 64)).astype(np.int64))
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    (a0, b0, t0, s0), (a1, b1, t1, s1) = out[0], out[1]
    assert a0 == 0 and b0 == a1 and b1 == len(sizes)
    assert t0 == t1 == float(sum(sizes))
    assert s0 == s1 == 11.0
    n0, n1 = sum(sizes[a0:b0]), sum(sizes[a1:b1])
    assert abs(n0 - n1) <= max(sizes)


def test_shard_edge_cases():
    assert sbh_dist.shard_systems([], 4, 2) == (0, 0)
    assert sbh_dist.shard_systems([5], 1, 0) == (0, 1)
    parts = [sbh_dist.shard_systems([3, 3, 3], 4, r) for r in range(4)]
    covered = [i for a, b in parts for i in range(a, b)]
    assert covered == [0, 1, 2]
    np.testing.assert_array_equal(sbh_dist.system_offsets([2, 3]), [0, 2, 5])


class _ShareTree:
    """CPU stand-in for a NativeTree on one rank: force rows are the target
    index inside the rank's target range and zero outside; the gradient is a
    partial sum over the rank's targets, spread over every particle."""

    def __init__(self, n):
        import torch

        self.n = n
        self.range = (0, n)
        self.torch = torch

    def set_target_range(self, b, e):
        assert 0 <= b <= e <= self.n
        self.range = (b, e)

    def _force(self):
        t = self.torch
        f = t.zeros((self.n, 3))
        b, e = self.range
        f[b:e] = t.arange(b, e, dtype=t.float32)[:, None]
        return f

    def force(self, **kw):
        return self._force()

    def force_vjp(self, cot, want_force=True, **kw):
        t = self.torch
        b, e = self.range
        share = float(cot[b:e].sum())
        gx = t.full((self.n, 3), share)
        gm = t.full((self.n,), float(e - b))
        return (self._force() if want_force else None), gx, gm


def _target_worker(rank, world, port, n, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    tree = _ShareTree(n)
    cot = torch.arange(n * 3, dtype=torch.float32).reshape(n, 3) / n
    f, gx, gm = sbh_dist.sharded_force_vjp(tree, cot)
    f2 = sbh_dist.sharded_force(tree)
    out[rank] = (f.numpy().copy(), gx.numpy().copy(), gm.numpy().copy(), f2.numpy().copy(), tree.range)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_target_sharding_sums_to_full():
    """sharded_force_vjp / sharded_force: each rank serves its share of the
    targets, the all-reduce gives every rank the full force and gradient, and
    the target range is restored afterwards."""
    n = 1001
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_target_worker, args=(r, 2, port, n, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    full_f = np.repeat(np.arange(n, dtype=np.float32)[:, None], 3, axis=1)
    cot_sum = float((np.arange(n * 3, dtype=np.float32) / n).sum())
    for r in range(2):
        f, gx, gm, f2, rng = out[r]
        np.testing.assert_array_equal(f, full_f)
        np.testing.assert_array_equal(f2, full_f)
        np.testing.assert_allclose(gx, cot_sum, rtol=1e-5)
        np.testing.assert_array_equal(gm, float(n))
        assert rng == (0, n)


def test_shard_targets_partition():
    for n in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            parts = [sbh_dist.shard_targets(n, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            assert max(b - a for a, b in parts) - min(b - a for a, b in parts) <= 1
