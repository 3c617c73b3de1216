"""The multi-rank timing of bench.py on CPU: two gloo ranks, the slowest
rank's figure wins (the device-time reduction the GPU runs use over NCCL)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.reduce_max([1.0 + rank, 10.0 - rank, 5.0], dist, "cpu")
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_reduce_max_over_two_gloo_ranks():
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res[0] == res[1] == [2.0, 10.0, 5.0]


def test_reduce_max_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max([3, 1.5]) == [3.0, 1.5]
