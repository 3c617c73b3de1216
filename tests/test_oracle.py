"""The CPU restatement (oracle/) pinned against the reference.

* every golden fixture (containers written by the reference's own
  compressor, tests/golden/) is reproduced byte for byte and decodes back;
* when the reference binaries built here from its sources are present
  (oracle/_ref), extra seeded cases are compared against them directly;
* the derived tables satisfy the reference's construction
  (cucm_compress_v2.cu:681-705) and the order-0/1 slot sets are
  collision-free, which the compact device layout relies on.
"""
import hashlib
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from tests.golden.golden_inputs import CASES, make_input

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("entry", _manifest(), ids=lambda e: e["name"])
def test_oracle_matches_golden(oracle_mod, entry):
    data = make_input(entry)
    assert hashlib.sha256(data).hexdigest() == entry["input_sha256"]
    with open(os.path.join(GOLDEN, entry["name"] + ".cucm"), "rb") as f:
        golden = f.read()
    assert hashlib.sha256(golden).hexdigest() == entry["output_sha256"]
    got = oracle_mod.compress(data, entry["chunksize"], entry["unit"], entry["prelearn"], entry["batch"], threads=4)
    assert got == golden
    assert oracle_mod.decompress(golden, threads=4) == data


def test_manifest_covers_cases():
    names = {e["name"] for e in _manifest()}
    assert names == {c["name"] for c in CASES}


def _ref(name):
    from oracle import ref_binary
    return ref_binary(name)


@pytest.mark.skipif(_ref("cucm_compress_ref") is None, reason="reference binaries not built here")
@pytest.mark.parametrize("kind,size,cs,unit,pre,batch", [
    ("text", 50001, 8192, 128, 0, 3),
    ("walk", 30000, 5000, 64, 0, 100),
    ("runs", 40000, 16384, 160, 4000, 2),
    ("random", 7000, 2048, 32, 0, 1),
])
def test_oracle_matches_reference_binary(oracle_mod, kind, size, cs, unit, pre, batch):
    data = make_input(dict(kind=kind, size=size, seed=size))
    with tempfile.TemporaryDirectory() as tmp:
        src, dst = os.path.join(tmp, "in"), os.path.join(tmp, "out")
        with open(src, "wb") as f:
            f.write(data)
        cmd = [_ref("cucm_compress_ref"), "-f", src, "-o", dst, "-s", str(cs), "-u", str(unit), "-b", str(batch)]
        if pre:
            cmd += ["-p", str(pre)]
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
        with open(dst, "rb") as f:
            ref = f.read()
    assert oracle_mod.compress(data, cs, unit, pre, batch, threads=4) == ref


def test_tables_follow_construction(oracle_mod):
    sq, st, dt, nex = oracle_mod.tables()
    knots = [1, 2, 3, 6, 10, 16, 27, 45, 73, 120, 194, 310, 488, 747, 1101, 1546, 2047, 2549, 2994, 3348, 3607,
             3785, 3901, 3975, 4022, 4050, 4068, 4079, 4085, 4089, 4092, 4093, 4094]
    for k in range(4095):
        d = k - 2047
        w, seg = d & 127, (d >> 7) + 16
        assert sq[k] == (knots[seg] * (128 - w) + knots[seg + 1] * w + 64) >> 7
    assert sq[4095] == 4095
    # stretch is the smallest x with squash(x) >= p
    for p in range(4095):
        x = st[p]
        assert sq[x + 2047] >= p and (x == -2047 or sq[x + 2046] < p)
    assert st[4095] == 2047
    assert list(dt) == [16384 // (2 * i + 3) for i in range(1024)]
    # 253 live bit-history states; rows 253..255 are empty
    assert nex.max() <= 252 and (nex[253:] == 0).all()


def test_low_orders_collision_free():
    basis, prime, mask = 2166136261, 16777619, (1 << 25) - 1
    o0 = {((basis ^ h0) * prime) & mask for h0 in range(1, 256)}
    assert len(o0) == 255
    o1 = set()
    for h0 in range(1, 256):
        a = ((basis ^ h0) * prime) & 0xFFFFFFFF
        for c in range(256):
            o1.add(((a ^ c) * prime) & mask)
    assert len(o1) == 255 * 256
