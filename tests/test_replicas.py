"""Multi-process host logic of the replica layout, world size 2 over gloo on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from slsimlib_b200.replicas import max_over_ranks, shard


def test_shard_covers_every_ray_once():
    for n in (0, 1, 7, 1000, 4_194_304):
        for world in (1, 2, 3, 8):
            ranges = [shard(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            for (a, b), (c, d) in zip(ranges, ranges[1:]):
                assert b == c
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    lo, hi = shard(4096, rank, world)
    slowest = max_over_ranks(10.0 + rank)  # rank 1 is the slowest
    dist.barrier()
    q.put((rank, lo, hi, slowest))
    dist.destroy_process_group()


def test_two_rank_gloo_timing_and_shards():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1:3] == (0, 2048) and out[1][1:3] == (2048, 4096)
    assert out[0][3] == out[1][3] == 11.0
