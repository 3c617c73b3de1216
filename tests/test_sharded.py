"""The multi-GPU split of one stream (cucm_b200/sharded.py), run as two and
three gloo ranks on the CPU.

Each rank codes its contiguous chunk range; the body sizes are all-gathered,
the bodies sent to rank 0 and framed there with the library's host framing
(cucm_frame_bodies); then rank 0 broadcasts the container, every rank decodes
its range and sends it back.  On the GPU the coder is libcucm on the rank's
device (DeviceCoder) over NCCL; here the ranks code and decode their
chunks with the oracle, so the test checks the split, the exchange steps and
the framing: the assembled container must equal the oracle's single-process
container byte for byte, and the round trip must give the stream back.
"""
import multiprocessing as mp
import os
import socket

import pytest

from cucm_b200 import sharded


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class HostCoder:
    """Chunk coding by the oracle (test infrastructure), framing by the library."""

    def __init__(self):
        import torch
        self.device = torch.device("cpu")

    def encode(self, block, chunksize, unit):
        import torch
        import oracle
        data = block.numpy().tobytes()
        if not data:
            return torch.empty(0, dtype=torch.uint8)
        blob = oracle.compress(data, chunksize, unit, 0, 65535)
        return torch.frombuffer(bytearray(blob[25:]), dtype=torch.uint8)

    def frame(self, params, orig_size, bodies, counts):
        import torch
        import cucm_b200
        blob = cucm_b200.frame_bodies([b.numpy().tobytes() for b in bodies], counts, orig_size,
                                      params.chunksize, params.unit, params.batch)
        return torch.frombuffer(bytearray(blob), dtype=torch.uint8)

    def decode_range(self, container, first, count, nbytes):
        import torch
        import oracle
        raw = container.numpy().tobytes()
        full = oracle.decompress(raw)
        cs = int.from_bytes(raw[8:12], "big")
        piece = full[first * cs:first * cs + nbytes]
        return torch.frombuffer(bytearray(piece), dtype=torch.uint8) if piece else torch.empty(0, dtype=torch.uint8)


def _rank(rank, world, port, data, cs, unit, batch, q):
    import datetime
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle")]
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n = len(data)
        first, count = sharded.split_chunks((n + cs - 1) // cs, world)[rank]
        lo, hi = first * cs, min(n, (first + count) * cs)
        block = torch.frombuffer(bytearray(data[lo:hi] or b"\0"), dtype=torch.uint8)[:max(0, hi - lo)]
        coder = HostCoder()
        container = sharded.compress_sharded(coder, block, n, cs, unit, batch, dist=dist)
        back = sharded.decompress_sharded(coder, container, n, cs, dist=dist)
        if rank == 0:
            q.put((container.numpy().tobytes(), back.numpy().tobytes()))
    finally:
        dist.destroy_process_group()


def test_split_chunks():
    assert sharded.split_chunks(10, 3) == [(0, 4), (4, 3), (7, 3)]
    assert sharded.split_chunks(2, 4) == [(0, 1), (1, 1), (2, 0), (2, 0)]
    assert sharded.split_chunks(0, 2) == [(0, 0), (0, 0)]


@pytest.mark.parametrize("world,size,cs,unit,batch", [
    (2, 40000, 4096, 128, 3),     # 10 chunks, batches of 3 straddle the ranks, partial last chunk
    (3, 24576, 4096, 64, 100),    # whole chunks only
    (2, 5000, 4096, 128, 1),      # the second rank holds only the short last chunk
])
def test_sharded_round_trip_equals_single(oracle_mod, cucm_lib, world, size, cs, unit, batch):
    from cucm_b200 import workloads as W
    data = W.text(size, size).tobytes()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, data, cs, unit, batch, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        container, back = q.get(timeout=180)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert container == oracle_mod.compress(data, cs, unit, 0, batch)
    assert back == data
