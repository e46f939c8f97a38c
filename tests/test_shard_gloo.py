"""Multi-rank host logic of the data-parallel path, on CPU with gloo
(world_size 2 and 3): shards tile the batch exactly once and the step time
reported is the max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from shrinkage_full_tests_b200.shard import batch_shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, B, q):
    import torch
    import torch.distributed as dist
    from shrinkage_full_tests_b200.shard import batch_shard, max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    start, count = batch_shard(B, rank, world)
    mine = torch.zeros(B, dtype=torch.int64)
    mine[start:start + count] = 1
    dist.all_reduce(mine)
    t = max_over_ranks(1.0 + rank, dist)
    q.put((rank, mine.tolist(), t))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,B", [(2, 5000), (3, 7)])
def test_batch_shards_cover_once_and_time_is_max(world, B):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, B, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, cover, t in res:
        assert cover == [1] * B
        assert t == float(world)


def test_batch_shard_edges():
    assert batch_shard(10, 0, 3) == (0, 4)
    assert batch_shard(10, 2, 3) == (7, 3)
    assert batch_shard(0, 0, 2) == (0, 0)
    with pytest.raises(ValueError):
        batch_shard(5, 2, 2)
