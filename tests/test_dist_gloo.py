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
