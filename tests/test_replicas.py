"""Multi-process host logic of the replica layout (bench.py --gpus N), world
size 2 over gloo on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from slsimlib_b200.replicas import max_over_ranks


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
    slowest = max_over_ranks(10.0 + rank)  # rank 1 is the slowest
    dist.barrier()
    q.put((rank, slowest))
    dist.destroy_process_group()


def test_two_rank_gloo_timing():
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
    assert out[0][1] == out[1][1] == 11.0
