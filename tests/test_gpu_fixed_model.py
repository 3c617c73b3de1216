"""The fixed-model variant on the GPU: containers equal the oracle's (which
defines this variant's stream; the reference has no code for it) byte for
byte and decode back, in the single call and the batched form; the serving
loop refuses the variant."""
import pytest

import cucm_b200 as cc
from cucm_b200 import workloads as W

pytestmark = pytest.mark.gpu

CASES = [("text", 300000, 65536, 20000), ("walk", 200000, 32768, 4000), ("runs", 70000, 16384, 16384),
         ("random", 50000, 8192, 1000), ("text", 9000, 262144, 3000)]


@pytest.mark.parametrize("kind,size,cs,pre", CASES)
def test_fixed_matches_oracle(gpu_ctx, oracle_mod, kind, size, cs, pre):
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    data = W.make(kind, size, size + 3).tobytes()
    want = oracle_mod.compress(data, cs, 128, pre, 100, fixed=True)
    got = gpu_ctx.compress(data, cs, 128, pre, 100, fixed=True)
    assert got == want
    assert gpu_ctx.decompress(want) == data


def test_fixed_batched_and_64bit(gpu_ctx, oracle_mod):
    bufs = [W.make(k, s, s).tobytes() for k, s in (("text", 40000), ("walk", 25000), ("text", 6000))]
    want = [oracle_mod.compress(b, 8192, 128, 2000, 100, fixed=True) for b in bufs]
    assert gpu_ctx.compress_many(bufs, chunksize=8192, prelearn=2000) != want  # adaptive by default
    got = [gpu_ctx.compress(b, 8192, 128, 2000, 100, fixed=True) for b in bufs]
    assert got == want
    assert gpu_ctx.decompress_many(want) == bufs
    wide = gpu_ctx.compress(bufs[0], 8192, 128, 2000, 100, fmt=cc.FORMAT_64, fixed=True)
    assert gpu_ctx.decompress(wide) == bufs[0]


def test_serving_loop_refuses_fixed(oracle_mod):
    data = W.text(20000, 2).tobytes()
    blob = oracle_mod.compress(data, 8192, 128, 2000, 100, fixed=True)
    with cc.Server(0, hbm_budget=8 << 30) as srv:
        st, _, _ = srv.poll(srv.submit_decompress(blob), -1)
        assert st == cc.EINVAL
