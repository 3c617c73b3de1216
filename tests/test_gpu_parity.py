"""GPU parity: the CUDA path against the oracle and the reference's goldens.

The bar is byte identity.  Compressed containers must equal the oracle's
(which tests/test_oracle.py pins to the reference) and the reference's own
golden outputs; decompression must reproduce the input exactly (the
full-size workloads are pinned in test_gpu_fullsize.py).  Every
execution choice (launch form, decoder speculation depth) must leave the
bytes unchanged.  All calls go through the C ABI (libcucm.so).
"""
import hashlib
import json
import os

import numpy as np
import pytest

import cucm_b200 as cc
from cucm_b200 import workloads as W
from tests.golden.golden_inputs import make_input

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(GOLDEN, "manifest.json")) as _f:
    MANIFEST = json.load(_f)


@pytest.mark.parametrize("entry", MANIFEST, ids=lambda e: e["name"])
@pytest.mark.parametrize("form", [cc.FORM_PERSISTENT, cc.FORM_PLAIN], ids=["persistent", "plain"])
def test_golden_compress(gpu_ctx, entry, form):
    gpu_ctx.set_tuning(form=form)
    data = make_input(entry)
    with open(os.path.join(GOLDEN, entry["name"] + ".cucm"), "rb") as f:
        golden = f.read()
    got = gpu_ctx.compress(data, entry["chunksize"], entry["unit"], entry["prelearn"], entry["batch"])
    assert hashlib.sha256(got).hexdigest() == entry["output_sha256"]
    assert got == golden


# decoders: the warp-pair kernel (units <= 256), and the generic kernel at
# three speculation depths
DECODERS = [(0, 0), (1, 1), (1, 4), (1, 8)]


@pytest.mark.parametrize("entry", MANIFEST, ids=lambda e: e["name"])
@pytest.mark.parametrize("kernel,spec", DECODERS, ids=["pair", "generic1", "generic4", "generic8"])
def test_golden_decompress(gpu_ctx, entry, kernel, spec):
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT, spec_bits=spec, kernel=kernel)
    with open(os.path.join(GOLDEN, entry["name"] + ".cucm"), "rb") as f:
        golden = f.read()
    assert gpu_ctx.decompress(golden) == make_input(entry)


CASES = [
    ("text", 300000, 65536, 128, 0, 100),
    ("walk", 200000, 32768, 128, 0, 3),
    ("runs", 150000, 65536, 64, 0, 100),
    ("random", 70000, 16384, 256, 0, 2),
    ("text", 60000, 16384, 160, 0, 100),      # units of 160..224 bits: 8 keys per lane, padded
    ("walk", 50000, 8192, 224, 0, 5),
    ("text", 100000, 10000, 96, 20000, 100),
    ("text", 65536 * 3, 65536, 128, 0, 1),
    ("walk", 12345, 1000, 32, 0, 7),
    ("text", 5000, 262144, 128, 0, 100),      # one tiny chunk with a long stale tail
    ("runs", 100000, 8192, 1024, 0, 100),     # largest unit
]


@pytest.mark.parametrize("kind,size,cs,unit,pre,batch", CASES)
@pytest.mark.parametrize("form", [cc.FORM_PERSISTENT, cc.FORM_PLAIN], ids=["persistent", "plain"])
def test_against_oracle(gpu_ctx, oracle_mod, kind, size, cs, unit, pre, batch, form):
    gpu_ctx.set_tuning(form=form)
    data = W.make(kind, size, size + cs).tobytes()
    want = oracle_mod.compress(data, cs, unit, pre, batch)
    got = gpu_ctx.compress(data, cs, unit, pre, batch)
    assert got == want
    assert gpu_ctx.decompress(want) == data
    gpu_ctx.set_tuning(form=form, kernel=1)
    assert gpu_ctx.decompress(want) == data


def test_speculation_depth_never_changes_output(gpu_ctx, oracle_mod):
    data = W.text(120000, 11).tobytes()
    blob = oracle_mod.compress(data, 32768, 128, 0, 100)
    for spec in range(1, 9):
        gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT, spec_bits=spec, kernel=1)
        assert gpu_ctx.decompress(blob) == data
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT, kernel=0)
    assert gpu_ctx.decompress(blob) == data


def test_batch_helpers_match_container(gpu_ctx, oracle_mod):
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    data = W.walk(50000, 4).tobytes()
    body = gpu_ctx.compress_batch(data, 8192, 128)
    full = oracle_mod.compress(data, 8192, 128, 0, 100)
    # container = 21-byte header + u32 LE batch size + batch body
    assert full[25:] == body
    assert int.from_bytes(full[21:25], "little") == len(body)
    assert gpu_ctx.decompressbatch(body, len(data), 8192, 128) == data


def test_config0_roundtrip_and_oracle(gpu_ctx, oracle_mod):
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    data, p = W.config0()
    data = data.tobytes()
    got = gpu_ctx.compress(data, **p)
    assert got == oracle_mod.compress(data, **p)
    assert gpu_ctx.decompress(got) == data


def test_many_equals_single(gpu_ctx):
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    bufs = [W.make(k, s, i).tobytes() for i, (k, s) in
            enumerate([("text", 40000), ("runs", 3000), ("walk", 70000), ("random", 20000), ("text", 1)])]
    many = gpu_ctx.compress_many(bufs, chunksize=16384)
    single = [gpu_ctx.compress(b, chunksize=16384) for b in bufs]
    assert many == single
    assert gpu_ctx.decompress_many(many) == bufs


def test_bad_container_rejected(gpu_ctx):
    with pytest.raises(cc.CucmError):
        gpu_ctx.decompress(b"\x00\x00\x10\x00" + bytes(10))
    blob = bytearray(gpu_ctx.compress(b"hello world" * 100, chunksize=256))
    with pytest.raises(cc.CucmError):
        gpu_ctx.decompress(bytes(blob[:30]))


@pytest.mark.parametrize("name", ["text_12k_pre3000", "random_12k_pre2000"])
def test_batch_bodies_of_prelearned_container(gpu_ctx, name):
    """compress_batch / decompressbatch with the reference's sm_init and
    mixer_init: a prelearned container's batch body is the batch coded from
    the container's model, and decodes back through it."""
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    entry = next(e for e in MANIFEST if e["name"] == name)
    data = make_input(entry)
    with open(os.path.join(GOLDEN, name + ".cucm"), "rb") as f:
        golden = f.read()
    pre = entry["prelearn"]
    coded = int.from_bytes(golden[12:16], "big")
    pl_len = coded if golden[20] else pre
    at = 21 + pl_len
    body = golden[at + 4:at + 4 + int.from_bytes(golden[at:at + 4], "little")]
    rest = data[pre:]
    for model in (cc.Model.from_container(golden), cc.Model.prelearn(data[:pre])):
        assert gpu_ctx.compress_batch(rest, entry["chunksize"], entry["unit"], model=model) == body
        assert gpu_ctx.decompressbatch(body, len(rest), entry["chunksize"], entry["unit"], model=model) == rest
    # the zero model gives a different body for the same bytes
    assert gpu_ctx.compress_batch(rest, entry["chunksize"], entry["unit"]) != body
