"""The 64-bit container on the GPU.

* Small streams written with CUCM_FORMAT_64 (with and without a prelearn
  prefix) hold the same chunk payloads as the reference's 32-bit container
  (the oracle's) and decode back, through the single call and the batched
  form;
* a stream past 4 GiB -- which the reference's 32-bit fields cannot describe
  (cucm_compress_v2.cu:1197-1216, :1241) -- is written in the 64-bit
  container automatically and round-trips byte for byte.
"""
import numpy as np
import pytest

import cucm_b200 as cc
from cucm_b200 import workloads as W
from tests.test_container64 import _payloads32, _payloads64

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("size,cs,batch", [(150000, 16384, 3), (70000, 65536, 100)])
def test_small_streams_in_the_64bit_container(gpu_ctx, oracle_mod, size, cs, batch):
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    data = W.make("walk", size, size).tobytes()
    v2 = gpu_ctx.compress(data, cs, 128, 0, batch, fmt=cc.FORMAT_64)
    _, _, _, _, pays = _payloads64(v2)
    assert pays == _payloads32(oracle_mod.compress(data, cs, 128, 0, batch), cs)
    assert gpu_ctx.decompress(v2) == data
    assert gpu_ctx.decompress_many([v2, v2[:]]) == [data, data]


def test_prelearn_in_the_64bit_container(gpu_ctx, oracle_mod):
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    data = W.text(60000, 5).tobytes()
    v1 = gpu_ctx.compress(data, 8192, 128, 6000, 100)
    assert v1 == oracle_mod.compress(data, 8192, 128, 6000, 100)
    v2 = gpu_ctx.compress(data, 8192, 128, 6000, 100, fmt=cc.FORMAT_64)
    # same prelearn block and payloads behind the wider header
    coded = int.from_bytes(v1[12:16], "big")
    pl = coded if v1[20] else 6000
    assert v2[45:45 + pl] == v1[21:21 + pl]
    assert gpu_ctx.decompress(v2) == data


def test_stream_past_4gib_round_trip(gpu_ctx):
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    block = W.config1(total=64 << 20)[0]
    data = np.tile(block, 64)  # 4 GiB
    data = np.concatenate([data, block[:3 << 20]])  # + 3 MiB
    n = data.size
    assert n > 0xFFFFFFFF
    blob = gpu_ctx.compress(data, chunksize=1 << 20, out=np.empty(n, dtype=np.uint8))  # the mix codes to ~0.6
    assert blob[:8].tobytes() == b"\xff\xff\xff\xff\x00\x00\x00\x02"
    assert int.from_bytes(blob[8:16].tobytes(), "big") == n
    back = gpu_ctx.decompress(blob, out=np.empty(n, dtype=np.uint8))
    assert back.size == n
    assert np.array_equal(back, data)
