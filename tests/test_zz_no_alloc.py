"""cucm_compress_chunk_noalloc: the compress entry point that allocates nothing.

It serves callers that cannot allocate device memory while they compress:
plugins inside a host application that owns every device allocation through
its own memory manager, and paths that cannot afford cudaMalloc's implicit
device synchronisation.  Its only scratch is a file-scope device array holding one
chunk's tables, shared by every call.  This test calls it through the C ABI
twice in a row on the same inputs -- the second call finds the first call's
tables in that array and must start from clean ones -- and checks each
result byte for byte against the chunk payload of the regular entry point
(cucm_compress_batch).  The buffers are the test's own (torch); the entry
point allocates nothing.
"""
import ctypes

import pytest

import cucm_b200 as cc
from cucm_b200 import workloads as W

pytestmark = pytest.mark.gpu

CASES = [
    ("text", 60000, 65536, 128),    # shorter than its chunk: stale tail coded to the chunk end
    ("walk", 32768, 32768, 128),    # exactly one chunk
    ("runs", 20000, 20000, 64),
    ("random", 9000, 16384, 256),
]


def _noalloc(lib, d_in, n, cs, unit, d_out, cap):
    got = ctypes.c_uint64()
    rc = lib.cucm_compress_chunk_noalloc(d_in, n, cs, unit, d_out, cap, ctypes.byref(got), None)
    return rc, got.value


@pytest.mark.parametrize("kind,size,cs,unit", CASES)
def test_noalloc_matches_regular_entry_point(kind, size, cs, unit):
    import torch

    lib = cc.lib()
    data = W.make(kind, size, size + unit).tobytes()
    with cc.Context(0) as ctx:
        body = ctx.compress_batch(data, cs, unit)  # [big-endian end offset][payload]
    want = body[4:]
    d_in = torch.tensor(list(data), dtype=torch.uint8, device="cuda")
    cap = 32 * cs + 16
    d_out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    for _ in range(2):
        d_out.fill_(0xAA)
        torch.cuda.synchronize()
        rc, n = _noalloc(lib, d_in.data_ptr(), len(data), cs, unit, d_out.data_ptr(), cap)
        assert rc == 0, cc.lib().cucm_strerror(rc)
        assert n == len(want)
        assert bytes(d_out[:n].cpu().numpy().tobytes()) == want


def test_noalloc_limits():
    import torch

    lib = cc.lib()
    data = W.text(5000, 3).tobytes()
    d_in = torch.tensor(list(data), dtype=torch.uint8, device="cuda")
    d_out = torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    # more than one chunk: the scratch holds one chunk's tables
    assert _noalloc(lib, d_in.data_ptr(), 5000, 4096, 128, d_out.data_ptr(), 1 << 20)[0] == -1
    assert _noalloc(lib, d_in.data_ptr(), 5000, 8192, 48, d_out.data_ptr(), 1 << 20)[0] == -1
    assert _noalloc(lib, d_in.data_ptr(), 5000, 8192, 512, d_out.data_ptr(), 1 << 20)[0] == -1
    # output too small: reports the size it needs
    rc, need = _noalloc(lib, d_in.data_ptr(), 5000, 8192, 128, d_out.data_ptr(), 16)
    assert rc == -2 and need > 16
    rc, n = _noalloc(lib, d_in.data_ptr(), 5000, 8192, 128, d_out.data_ptr(), need)
    assert rc == 0 and n == need
