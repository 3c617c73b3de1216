"""The full-size benchmark workloads, pinned byte for byte against the reference.

tests/golden/fullsize_manifest.json holds the SHA-256 of the containers the
reference's own code writes for them (tests/golden/make_fullsize.py runs the
reference's compressor, built from its sources, on the host):

* the 256 MiB mixed buffer at 1 MiB chunks (256 chunks): the container from
  the persistent form and from the plain form (one launch per chunk) must
  both hash to the reference's, and decode back to the input;
* the 4096 buffers of log-uniform size at 256 KiB chunks: every container of
  the batched persistent form must hash to the reference's and decode back;
  the plain form codes a stratified sample of 512 buffers (every 8th buffer in
  size order, the smallest and the largest included) to the same hashes.
"""
import hashlib
import json
import os

import pytest

import cucm_b200 as cc
from cucm_b200 import workloads as W

pytestmark = pytest.mark.gpu

MANIFEST = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fullsize_manifest.json")
with open(MANIFEST) as _f:
    MAN = json.load(_f)


def _sha(b):
    return hashlib.sha256(b).hexdigest()


def test_mixed256m_matches_reference(gpu_ctx):
    data, p = W.config1()
    m = MAN["mixed256M"]
    assert _sha(data.tobytes()) == m["input_sha256"]
    blob = None
    for form in (cc.FORM_PERSISTENT, cc.FORM_PLAIN):
        gpu_ctx.set_tuning(form=form)
        blob = gpu_ctx.compress(data, **p)
        assert len(blob) == m["output_len"]
        assert _sha(blob) == m["output_sha256"], form
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    assert gpu_ctx.decompress(blob) == data.tobytes()


@pytest.fixture(scope="module")
def many4096():
    bufs, p = W.config2()
    m = MAN["many4096"]
    assert [len(b) for b in bufs] == m["input_lens"]
    return bufs, p, m


def test_many4096_batched_matches_reference(gpu_ctx, many4096):
    bufs, p, m = many4096
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    blobs = gpu_ctx.compress_many(bufs, **p)
    bad = [i for i, b in enumerate(blobs) if _sha(b) != m["output_sha256"][i]]
    assert not bad, "containers differing from the reference: %s" % bad[:10]
    back = gpu_ctx.decompress_many(blobs)
    assert all(x == y.tobytes() for x, y in zip(back, bufs))


def test_many4096_plain_sample_matches_reference(gpu_ctx, many4096):
    bufs, p, m = many4096
    pick = W.config2_sample(512)
    lens = m["input_lens"]
    assert len(pick) == 512
    assert min(lens[i] for i in pick) == min(lens) and max(lens[i] for i in pick) == max(lens)
    gpu_ctx.set_tuning(form=cc.FORM_PLAIN)
    blobs = gpu_ctx.compress_many([bufs[i] for i in pick], **p)
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    bad = [i for i, b in zip(pick, blobs) if _sha(b) != m["output_sha256"][i]]
    assert not bad, "containers differing from the reference: %s" % bad[:10]
