"""The serving loop: continuous batching of mixed compress / decompress
requests.  Each result must be byte-identical whether its request ran alone
or in a mix of concurrent requests (the tolerance is zero: the bar is byte
identity), and equal to the single-call API's output.  A small slot pool
forces requests to wait for slots and be admitted while others run."""
import numpy as np
import pytest

import cucm_b200 as cc
from cucm_b200 import workloads as W

pytestmark = pytest.mark.gpu

CS = 65536


def _requests(seed, count=24):
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(1024), np.log(600000), size=count))).astype(int)
    kinds = rng.choice(4, size=count, p=[0.5, 0.25, 0.15, 0.10])
    ops = rng.random(count) < 0.7
    out = []
    for i, (n, k, comp) in enumerate(zip(sizes, kinds, ops)):
        data = W.make(W.KINDS[k], int(n), seed * 1000 + i).tobytes()
        out.append((bool(comp), data))
    return out


@pytest.fixture(scope="module")
def reqs_and_truth(gpu_ctx):
    gpu_ctx.set_tuning(form=cc.FORM_PERSISTENT)
    reqs = _requests(4)
    truth = []
    for comp, data in reqs:
        blob = gpu_ctx.compress(data, chunksize=CS)
        truth.append((blob, data))
    return reqs, truth


def _submit(srv, comp, data, blob):
    return srv.submit_compress(data, chunksize=CS) if comp else srv.submit_decompress(blob)


@pytest.mark.parametrize("max_slots", [0, 3], ids=["pool", "3slots"])
def test_mix_equals_alone(reqs_and_truth, max_slots):
    reqs, truth = reqs_and_truth
    with cc.Server(0, hbm_budget=24 << 30, max_slots=max_slots) as srv:
        ids = [_submit(srv, comp, data, blob) for (comp, data), (blob, _) in zip(reqs, truth)]
        mix = [srv.poll(i, -1) for i in ids]
        alone = []
        for (comp, data), (blob, _) in zip(reqs, truth):
            alone.append(srv.poll(_submit(srv, comp, data, blob), -1))
        info = srv.stats()
    for (comp, data), (blob, _), m, a in zip(reqs, truth, mix, alone):
        want = blob if comp else data
        assert m[0] == 0 and a[0] == 0
        assert m[1] == want
        assert a[1] == want
        assert m[2] > 0 and a[2] > 0
    assert info["completed"] == 2 * len(reqs)
    assert info["queued"] == 0 and info["inflight"] == 0


def test_serve_errors(gpu_ctx):
    with cc.Server(0, hbm_budget=8 << 30) as srv:
        bad = srv.submit_decompress(b"\x00\x00\x10\x00" + bytes(30))
        st, data, _ = srv.poll(bad, -1)
        assert st == cc.EFORMAT and data is None
        # a too-small output buffer reports ENOSPC and the size needed
        data = W.make("random", 40000, 3).tobytes()
        small = np.zeros(100, dtype=np.uint8)
        rid = srv.submit_compress(data, chunksize=8192, out=small)
        st, _, _ = srv.poll(rid, -1)
        assert st == cc.ENOSPC
        with pytest.raises(cc.CucmError):
            srv.poll(123456789, 0)
        # prelearn requests carry their own model and still match the single call
        pre = W.make("text", 50000, 9).tobytes()
        rid = srv.submit_compress(pre, chunksize=8192, prelearn=3000)
        st, blob, _ = srv.poll(rid, -1)
        assert st == 0 and blob == gpu_ctx.compress(pre, chunksize=8192, prelearn=3000)
        rid = srv.submit_decompress(blob)
        st, back, _ = srv.poll(rid, -1)
        assert st == 0 and back == pre
