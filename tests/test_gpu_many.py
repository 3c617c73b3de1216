"""The batched form: many containers in one call, one persistent launch.

Each container must be byte-identical to what the single-buffer call makes
of the same buffer (and so to the reference, which tests/test_gpu_parity.py
pins), whatever the mix of sizes, content types, launch form and unit
lengths, and decompress_many must give every buffer back.  Host and device
entry points alike, through the C ABI.
"""
import ctypes

import numpy as np
import pytest

import cucm_b200 as cc
from cucm_b200 import workloads as W

pytestmark = pytest.mark.gpu

MIX = [("text", 40000), ("runs", 3000), ("walk", 70000), ("random", 20000), ("text", 1), ("runs", 0),
       ("text", 7), ("walk", 16384), ("random", 16385), ("text", 90001), ("runs", 120000), ("walk", 5)]


def _bufs(seed=0):
    return [W.make(k, s, seed * 100 + i).tobytes() for i, (k, s) in enumerate(MIX)]


@pytest.mark.parametrize("form", [cc.FORM_PERSISTENT, cc.FORM_PLAIN], ids=["persistent", "plain"])
def test_many_equals_single_and_oracle(gpu_ctx, oracle_mod, form):
    gpu_ctx.set_tuning(form=form)
    bufs = _bufs(1)
    many = gpu_ctx.compress_many(bufs, chunksize=16384)
    for b, m in zip(bufs, many):
        assert m == oracle_mod.compress(b, 16384, 128, 0, 100)
    assert gpu_ctx.decompress_many(many) == bufs


def test_many_small_batches_and_units(gpu_ctx, oracle_mod):
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    bufs = _bufs(2)
    a = gpu_ctx.compress_many(bufs[:6], chunksize=4096, unit=64, batch=3)
    b = gpu_ctx.compress_many(bufs[6:], chunksize=8192, unit=256, batch=2)
    for x, y in zip(bufs[:6], a):
        assert y == oracle_mod.compress(x, 4096, 64, 0, 3)
    for x, y in zip(bufs[6:], b):
        assert y == oracle_mod.compress(x, 8192, 256, 0, 2)
    # one decompress_many over containers of two unit lengths and chunk sizes
    mixed = a + b
    assert gpu_ctx.decompress_many(mixed) == bufs


def test_many_with_prelearn(gpu_ctx):
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    bufs = [W.make("text", 30000 + 1000 * i, 50 + i).tobytes() for i in range(4)]
    many = gpu_ctx.compress_many(bufs, chunksize=8192, prelearn=2000)
    assert many == [gpu_ctx.compress(b, chunksize=8192, prelearn=2000) for b in bufs]
    assert gpu_ctx.decompress_many(many) == bufs


def test_many_reports_short_output(gpu_ctx):
    """An entry whose output buffer is too small gets CUCM_ENOSPC and the
    size it needs; the other entries are still written."""
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    lib = cc.lib()
    bufs = [W.make("random", 30000, 7).tobytes(), W.make("text", 30000, 8).tobytes()]
    want = [gpu_ctx.compress(b, chunksize=8192) for b in bufs]
    p = cc.default_params(8192)
    k = 2
    ins_b = [ctypes.create_string_buffer(b, len(b)) for b in bufs]
    caps = [100, len(want[1]) + 10]
    outs_b = [ctypes.create_string_buffer(c) for c in caps]
    ins = (ctypes.c_void_p * k)(*[ctypes.addressof(x) for x in ins_b])
    ns = (ctypes.c_uint64 * k)(*[len(b) for b in bufs])
    outs = (ctypes.c_void_p * k)(*[ctypes.addressof(x) for x in outs_b])
    capa = (ctypes.c_uint64 * k)(*caps)
    got = (ctypes.c_uint64 * k)()
    st = (ctypes.c_int * k)()
    rc = lib.cucm_compress_many(gpu_ctx._h, k, ins, ns, ctypes.byref(p), outs, capa, got, st)
    assert rc == cc.ENOSPC
    assert st[0] == cc.ENOSPC and got[0] == len(want[0])
    assert st[1] == 0 and outs_b[1].raw[:got[1]] == want[1]


def test_many_dev_matches_host(gpu_ctx):
    import torch

    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    bufs = _bufs(3)
    want = gpu_ctx.compress_many(bufs, chunksize=16384)
    d_in = [torch.tensor(np.frombuffer(b, np.uint8).copy() if b else np.zeros(1, np.uint8), device="cuda")
            for b in bufs]
    caps = [cc.many_cap(len(b), 16384) for b in bufs]
    d_out = [torch.empty(c, dtype=torch.uint8, device="cuda") for c in caps]
    torch.cuda.synchronize()
    sizes, st = gpu_ctx.compress_many_dev([(t.data_ptr(), len(b)) for t, b in zip(d_in, bufs)],
                                          [(t.data_ptr(), c) for t, c in zip(d_out, caps)], chunksize=16384)
    assert st == [0] * len(bufs)
    got = [bytes(t[:n].cpu().numpy().tobytes()) for t, n in zip(d_out, sizes)]
    assert got == want
    back = [torch.empty(max(len(b), 1), dtype=torch.uint8, device="cuda") for b in bufs]
    sizes2, st2 = gpu_ctx.decompress_many_dev([(t.data_ptr(), n) for t, n in zip(d_out, sizes)],
                                              [(t.data_ptr(), len(b)) for t, b in zip(back, bufs)])
    assert st2 == [0] * len(bufs) and sizes2 == [len(b) for b in bufs]
    assert [bytes(t[:len(b)].cpu().numpy().tobytes()) for t, b in zip(back, bufs)] == bufs


def test_decoder_with_many_chunks_in_flight(gpu_ctx, oracle_mod):
    """More chunks in flight than two per SM: the decoder's CTAs then hold
    more than two chunks each and keep the order 0/1 tables in the slot tables
    instead of shared memory; both placements must give the same bytes."""
    buf = W.make("text", 400 * 1024 + 123, 77).tobytes()
    comp = gpu_ctx.compress(buf, chunksize=1024)
    assert comp == oracle_mod.compress(buf, 1024, 128, 0, 100)
    assert gpu_ctx.decompress(comp) == buf
    few = buf[:2 * 1024 + 5]
    assert gpu_ctx.decompress(gpu_ctx.compress(few, chunksize=1024)) == few
