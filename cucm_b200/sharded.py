"""One stream's chunks coded on several GPUs, one process per GPU.

The reference codes a stream on one GPU.  Its chunks are independent (each
starts from the same initial model, with no history before its first
byte), so a stream splits into contiguous chunk ranges, one per rank:

compress -- every rank codes its range into a batch body (chunk end offsets
  and payloads, cucm_compress_batch_dev); the body sizes are all-gathered,
  every rank sends its body to the owner (rank 0), and the owner frames the
  bodies into the container (cucm_frame_bodies_dev), byte-identical to the
  single-GPU cucm_compress of the whole stream;
decompress -- the owner broadcasts the container, every rank decodes its
  chunk range (cucm_decompress_range_dev) and sends the bytes back to the
  owner, which places them in stream order.

The exchange steps are torch.distributed collectives and point-to-point
transfers of device tensors (NCCL over NVLink between GPUs; gloo on the CPU
in the tests, with a host coder).  Every rank takes the same collective
steps in the same order.  No kernel of this library waits on another rank.
"""
import ctypes

from . import CucmError, default_params, lib

__all__ = ["split_chunks", "DeviceCoder", "compress_sharded", "decompress_sharded"]


def split_chunks(nchunks, world):
    """Contiguous chunk ranges (first, count), one per rank, as even as the
    count allows; earlier ranks take the extra chunks."""
    base, extra = divmod(nchunks, world)
    out, at = [], 0
    for r in range(world):
        c = base + (1 if r < extra else 0)
        out.append((at, c))
        at += c
    return out


class DeviceCoder:
    """The coder of the sharded path: libcucm on this rank's GPU.  Tensors
    are torch uint8 tensors on `device`."""

    def __init__(self, ctx, device):
        import torch
        self.ctx = ctx
        self.device = torch.device(device)

    def _empty(self, n):
        import torch
        return torch.empty(max(int(n), 1), dtype=torch.uint8, device=self.device)

    def encode(self, block, chunksize, unit):
        """Batch body of the chunks in `block` (the rank's range)."""
        n = block.numel()
        nch = (n + chunksize - 1) // chunksize
        cap = nch * (4 + 2 * chunksize + 4096) + 16
        while True:
            out = self._empty(cap)
            got = ctypes.c_uint64()
            rc = lib().cucm_compress_batch_dev(self.ctx._h, block.data_ptr(), n, chunksize, unit, None,
                                               out.data_ptr(), cap, ctypes.byref(got))
            if rc == -2 and got.value > cap:  # ENOSPC reports the size it needs
                cap = got.value
                continue
            if rc:
                raise CucmError(rc, "cucm_compress_batch_dev")
            return out[:got.value]

    def frame(self, params, orig_size, bodies, counts):
        k = len(bodies)
        ptrs = (ctypes.c_void_p * k)(*[b.data_ptr() for b in bodies])
        ns = (ctypes.c_uint64 * k)(*[b.numel() for b in bodies])
        cs = (ctypes.c_uint32 * k)(*counts)
        cap = 64 + 4 * ((sum(counts) + params.batch - 1) // params.batch) + sum(b.numel() for b in bodies)
        out = self._empty(cap)
        got = ctypes.c_uint64()
        rc = lib().cucm_frame_bodies_dev(self.ctx._h, ctypes.byref(params), orig_size, k, ptrs, ns, cs,
                                         out.data_ptr(), cap, ctypes.byref(got))
        if rc:
            raise CucmError(rc, "cucm_frame_bodies_dev")
        return out[:got.value]

    def decode_range(self, container, first, count, nbytes):
        out = self._empty(nbytes)
        got = ctypes.c_uint64()
        rc = lib().cucm_decompress_range_dev(self.ctx._h, container.data_ptr(), container.numel(), first, count,
                                             out.data_ptr(), nbytes, ctypes.byref(got))
        if rc:
            raise CucmError(rc, "cucm_decompress_range_dev")
        return out[:got.value]


def _sizes(dist, n, device):
    import torch
    world = dist.get_world_size()
    mine = torch.tensor([int(n)], dtype=torch.int64, device=device)
    all_ = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(all_, mine)
    return [int(t.item()) for t in all_]


def compress_sharded(coder, block, orig_size, chunksize=1 << 20, unit=128, batch=100, dist=None):
    """Code this rank's `block` (its contiguous chunk range of a stream of
    `orig_size` bytes, as split_chunks splits it) and assemble the container
    on rank 0.  Returns the container tensor on rank 0, None elsewhere."""
    import torch
    rank, world = dist.get_rank(), dist.get_world_size()
    body = coder.encode(block, chunksize, unit)
    sizes = _sizes(dist, body.numel(), coder.device)
    counts = [c for _, c in split_chunks((orig_size + chunksize - 1) // chunksize, world)]
    if rank == 0:
        bodies = [body]
        for r in range(1, world):
            t = torch.empty(max(sizes[r], 1), dtype=torch.uint8, device=coder.device)
            if sizes[r]:
                dist.recv(t, src=r)
            bodies.append(t[:sizes[r]])
        params = default_params(chunksize, unit, 0, batch)
        return coder.frame(params, orig_size, bodies, counts)
    if sizes[rank]:
        dist.send(body.contiguous(), dst=0)
    return None


def decompress_sharded(coder, container, orig_size, chunksize, dist=None):
    """Decode the stream whose container rank 0 holds; every rank decodes its
    chunk range.  Returns the stream's bytes on rank 0, None elsewhere."""
    import torch
    rank, world = dist.get_rank(), dist.get_world_size()
    n = torch.tensor([container.numel() if rank == 0 else 0], dtype=torch.int64, device=coder.device)
    dist.broadcast(n, src=0)
    buf = container if rank == 0 else torch.empty(int(n.item()), dtype=torch.uint8, device=coder.device)
    dist.broadcast(buf, src=0)
    ranges = split_chunks((orig_size + chunksize - 1) // chunksize, world)
    first, count = ranges[rank]
    lo = first * chunksize
    mine = coder.decode_range(buf, first, count, max(0, min(orig_size, (first + count) * chunksize) - lo))
    if rank == 0:
        out = torch.empty(max(orig_size, 1), dtype=torch.uint8, device=coder.device)
        out[:mine.numel()] = mine
        for r in range(1, world):
            f, c = ranges[r]
            a, b = f * chunksize, min(orig_size, (f + c) * chunksize)
            if b > a:
                piece = torch.empty(b - a, dtype=torch.uint8, device=coder.device)
                dist.recv(piece, src=r)
                out[a:b] = piece
        return out[:orig_size]
    if mine.numel():
        dist.send(mine.contiguous(), dst=0)
    return None
