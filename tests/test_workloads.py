"""Seeded synthetic workloads are deterministic and have the stated shapes."""
import numpy as np

from cucm_b200 import workloads as W


def test_text_deterministic_and_alphabet(cucm_lib):
    a = W.text(20000, 7)
    b = W.text(20000, 7)
    assert (a == b).all()
    allowed = set(range(0x20, 0x7F)) | {0x0A}
    assert set(np.unique(a).tolist()) <= allowed
    assert not (W.text(20000, 8) == a).all()


def test_walk_is_int32_random_walk():
    b = W.walk(4 * 1000, 3)
    x = np.frombuffer(b.tobytes(), dtype="<i4")
    assert x[0] == 0
    d = np.diff(x.astype(np.int64))
    assert abs(d.std() - 100) < 15


def test_runs_and_random():
    r = W.runs(100000, 1)
    changes = np.count_nonzero(np.diff(r.astype(int)))
    assert 300 < changes < 700  # mean run 200
    u = W.random_bytes(1 << 16, 2)
    assert len(np.unique(u)) == 256


def test_config2_sizes():
    sizes, kinds = W.config2_sizes()
    assert len(sizes) == 4096 and sizes.min() >= 4096 and sizes.max() <= 4 << 20
    frac = np.bincount(kinds, minlength=4) / 4096
    assert abs(frac[0] - 0.5) < 0.05 and abs(frac[3] - 0.1) < 0.03


def test_config1_small():
    data, p = W.config1(total=1 << 20)
    assert len(data) == 1 << 20 and p["chunksize"] == 1 << 20
