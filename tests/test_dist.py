"""The N>1 path's host logic on CPU: two gloo ranks shard the images (each
exactly once), and the timing/throughput reductions take the slowest rank's
time and the sum of all ranks' pixels."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from unblending_b200 import dist as D


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        images = list(range(7))
        mine = D.shard(images, rank, world)
        ms = 10.0 * (rank + 1)                     # rank 1 is the slow one
        pixels = 1000.0 * len(mine)
        value = D.throughput(pixels, ms)
        out.put((rank, mine, value, D.reduce_max(ms), D.reduce_sum(pixels)))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = [r[1] for r in results]
    assert sorted(shards[0] + shards[1]) == list(range(7)) and not set(shards[0]) & set(shards[1])
    for rank, mine, value, mx, total in results:
        assert mx == 20.0 and total == 7000.0
        assert value == pytest.approx(7000.0 / 0.020)


def test_single_process_reductions_are_identity():
    assert D.reduce_max(3.5) == 3.5 and D.reduce_sum(2.0) == 2.0
    assert D.shard([1, 2, 3], 0, 1) == [1, 2, 3]
