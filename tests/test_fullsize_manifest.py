"""The full-size SHA-256 manifest (tests/golden/fullsize_manifest.json) and
how it was made, checked without a GPU.

make_fullsize.py codes each 1 MiB chunk of the 256 MiB workload as a file of
its own with the reference and frames the payloads into one container.  That
is only valid because a chunk's payload depends on nothing but its own bytes,
the chunk size and the unit, and because the framing is the reference's:
here the same per-chunk framing, applied to the oracle's single-chunk
payloads, must rebuild the reference's multi-chunk golden containers exactly.
"""
import hashlib
import json
import os
import struct

import pytest

from cucm_b200 import workloads as W
from tests.golden import make_fullsize as MF
from tests.golden.golden_inputs import make_input

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return {e["name"]: e for e in json.load(f)}


@pytest.mark.parametrize("name", ["text_20k_cs4k", "text_20k_cs4k_b2", "text_8192_cs4096", "walk_16k_cs4k",
                                  "text_10k_cs1000", "random_9k_cs4k"])
def test_chunkwise_framing_rebuilds_golden(oracle_mod, name):
    e = _manifest()[name]
    data = make_input(e)
    cs = e["chunksize"]
    payloads = []
    for k in range(0, len(data), cs):
        one = oracle_mod.compress(data[k:k + cs], cs, e["unit"], 0, e["batch"])
        (body,) = struct.unpack("<I", one[21:25])
        assert len(one) == 25 + body
        payloads.append(one[29:])
    blob = MF.frame(len(data), cs, e["unit"], e["batch"], payloads)
    with open(os.path.join(GOLDEN, name + ".cucm"), "rb") as f:
        assert blob == f.read()


def test_manifest_shape():
    with open(MF.OUT) as f:
        man = json.load(f)
    m1, m2 = man["mixed256M"], man["many4096"]
    assert m1["chunks"] == 256 and len(m1["chunk_payload_lens"]) == 256
    assert m1["output_len"] == 21 + 3 * 4 + 4 * 256 + sum(m1["chunk_payload_lens"])
    sizes, _ = W.config2_sizes()
    assert m2["input_lens"] == [int(s) for s in sizes]
    assert len(m2["output_sha256"]) == len(sizes) == len(m2["output_len"])
    assert all(len(h) == 64 for h in m2["output_sha256"])


def test_manifest_input_mixed256m():
    with open(MF.OUT) as f:
        m1 = json.load(f)["mixed256M"]
    data, _ = W.config1()
    assert hashlib.sha256(data.tobytes()).hexdigest() == m1["input_sha256"]
