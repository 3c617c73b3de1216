"""Failure paths, made to happen without faulting the GPU.

* The decoder's two warps per chunk meet through a bounded wait; with the
  bound set to a single poll (cucm_tuning.dec_spin_limit = 1) the updating
  warp gives up, the kernel returns with an error status and the call
  reports CUCM_ETIMEOUT.  The same context then decodes correctly with the
  default bound: the CUDA context stays usable.
* Truncated or inconsistent containers (header, batch size field, chunk end
  offsets, payload) are refused with CUCM_EFORMAT by the host-side parser
  before any device work, and the context keeps working.
* The serving loop refuses what its HBM budget cannot hold: a budget too
  small for the buffer pool (CUCM_ENOMEM at creation), a request whose own
  buffers exceed the buffer budget (status CUCM_ENOMEM), and submissions
  beyond the queue limit (CUCM_EBUSY).
"""
import struct

import numpy as np
import pytest

import cucm_b200 as cc
from cucm_b200 import workloads as W

pytestmark = pytest.mark.gpu

ETIMEOUT, ENOMEM, EBUSY = -7, -4, -8


def test_decoder_wait_timeout_then_recovers(gpu_ctx):
    data = W.text(200_000, 21).tobytes()
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    blob = gpu_ctx.compress(data, chunksize=65536)
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT, dec_spin_limit=1)
    with pytest.raises(cc.CucmError) as e:
        gpu_ctx.decompress(blob)
    assert e.value.status == ETIMEOUT
    gpu_ctx.set_tuning(form=cc.FORM_PLAIN, dec_spin_limit=1)
    with pytest.raises(cc.CucmError) as e:
        gpu_ctx.decompress(blob)
    assert e.value.status == ETIMEOUT
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    assert gpu_ctx.decompress(blob) == data
    # a bound that is large but not the default still decodes
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT, dec_spin_limit=1 << 24)
    assert gpu_ctx.decompress(blob) == data
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)


def _batches(blob):
    """(offset, body size) of every batch of a container without prelearn."""
    pos, out = 21, []
    while pos < len(blob):
        (size,) = struct.unpack("<I", blob[pos:pos + 4])
        out.append((pos, size))
        pos += 4 + size
    return out


def test_truncated_and_inconsistent_containers(gpu_ctx):
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    data = W.walk(40_000, 5).tobytes()
    blob = gpu_ctx.compress(data, chunksize=4096, batch=3)
    (b0, s0), (b1, s1) = _batches(blob)[:2]
    bad = [
        blob[:20],                     # inside the header
        blob[:b0 + 2],                 # inside the first batch size field
        blob[:b0 + 4 + 6],             # inside the first chunk end-offset table
        blob[:b0 + 4 + s0 - 1],        # first batch's payload cut short
        blob[:b1 + 4 + 8],             # second batch's table cut short
        blob[:-1],                     # last payload one byte short
    ]
    # a batch size that claims more than the container holds
    grown = bytearray(blob)
    grown[b0:b0 + 4] = struct.pack("<I", s0 + len(blob))
    bad.append(bytes(grown))
    # chunk end offsets that run backwards
    swapped = bytearray(blob)
    t = b0 + 4
    swapped[t:t + 4], swapped[t + 4:t + 8] = blob[t + 4:t + 8], blob[t:t + 4]
    bad.append(bytes(swapped))
    for i, b in enumerate(bad):
        with pytest.raises(cc.CucmError) as e:
            gpu_ctx.decompress(b)
        assert e.value.status == cc.EFORMAT, i
    assert gpu_ctx.decompress(blob) == data


def test_server_budget_too_small():
    with pytest.raises(cc.CucmError) as e:
        cc.Server(0, hbm_budget=1 << 30)
    assert e.value.status == ENOMEM


def test_server_refuses_request_over_buffer_budget():
    # 2.5 GiB: 2 GiB of buffers, 2 chunk slots
    with cc.Server(0, hbm_budget=5 << 29) as srv:
        big = np.zeros(1 << 30, dtype=np.uint8)  # needs input + 2x scratch: over 2 GiB
        rid = srv.submit_compress(big, chunksize=1 << 20, out=np.zeros(64, dtype=np.uint8))
        st, data, _ = srv.poll(rid, -1)
        assert st == ENOMEM and data is None
        small = W.text(30_000, 3).tobytes()
        rid = srv.submit_compress(small, chunksize=8192)
        st, blob, _ = srv.poll(rid, -1)
        assert st == 0 and cc.Context(0).decompress(blob) == small
        info = srv.stats()
        assert info["queued"] == 0 and info["inflight"] == 0


def test_server_queue_limit():
    with cc.Server(0, hbm_budget=8 << 30) as srv:
        srv.set_queue_limit(0)
        with pytest.raises(cc.CucmError) as e:
            srv.submit_compress(b"abc" * 100, chunksize=4096)
        assert e.value.status == EBUSY
        srv.set_queue_limit(16)
        rid = srv.submit_compress(b"abc" * 100, chunksize=4096)
        st, blob, _ = srv.poll(rid, -1)
        assert st == 0 and blob
