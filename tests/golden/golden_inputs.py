"""Seeded inputs of the golden fixtures (shared by make_golden.py and the tests).

Inputs are rebuilt from (kind, size, seed) with numpy's PCG64 so that only
the reference's outputs need to be committed.  Kinds mirror the benchmark
content types at small sizes: word-like text, an int32 random walk, uniform
random bytes and byte runs.
"""
import numpy as np


def _text(n, seed):
    rng = np.random.default_rng(seed)
    words = [bytes(rng.integers(97, 123, size=int(rng.integers(1, 9))).astype(np.uint8)) for _ in range(300)]
    out = bytearray()
    while len(out) < n:
        out += words[int(rng.integers(0, 300))] + b" "
    return bytes(out[:n])


def _walk(n, seed):
    rng = np.random.default_rng(seed)
    m = (n + 3) // 4
    x = np.concatenate([[0], np.cumsum(np.rint(rng.normal(0, 100, size=max(m - 1, 0))))]).astype(np.int64)
    return (x & 0xFFFFFFFF).astype("<u4").tobytes()[:n]


def _random(n, seed):
    return np.random.default_rng(seed).integers(0, 256, size=n, dtype=np.uint8).tobytes()


def _runs(n, seed):
    rng = np.random.default_rng(seed)
    out = bytearray()
    while len(out) < n:
        out += bytes([int(rng.integers(0, 256))]) * int(rng.geometric(1 / 200.0))
    return bytes(out[:n])


KINDS = {"text": _text, "walk": _walk, "random": _random, "runs": _runs}


def make_input(case):
    return KINDS[case["kind"]](case["size"], case["seed"])


def _c(name, kind, size, seed, chunksize, unit=128, prelearn=0, batch=100):
    return dict(name=name, kind=kind, size=size, seed=seed, chunksize=chunksize, unit=unit, prelearn=prelearn,
                batch=batch)


CASES = [
    _c("text_20k_cs4k", "text", 20000, 1, 4096),
    _c("text_20k_cs4k_b2", "text", 20000, 1, 4096, batch=2),
    _c("text_10k_cs1000", "text", 10000, 2, 1000),
    _c("text_10k_u32", "text", 10000, 3, 1024, unit=32),
    _c("text_10k_u96", "text", 10000, 3, 4096, unit=96),
    _c("text_10k_u256", "text", 10000, 3, 4096, unit=256),
    _c("text_12k_pre3000", "text", 12000, 4, 4096, prelearn=3000),
    _c("random_12k_pre2000", "random", 12000, 4, 4096, prelearn=2000),
    _c("walk_16k_cs4k", "walk", 16384, 5, 4096),
    _c("random_9k_cs4k", "random", 9000, 6, 4096),
    _c("runs_16k_cs4k", "runs", 16384, 7, 4096),
    _c("text_1_cs4k", "text", 1, 8, 4096),
    _c("text_7_cs4k", "text", 7, 8, 4096),
    _c("text_9_cs8", "text", 9, 8, 8),
    _c("text_0_cs4k", "text", 0, 8, 4096),
    _c("text_4097_cs4096_u64", "text", 4097, 9, 4096, unit=64, batch=1),
    _c("text_8192_cs4096", "text", 8192, 10, 4096),
    # edge sizes around one unit (16 bytes at unit 128) and one chunk
    _c("text_8_cs4k", "text", 8, 11, 4096),
    _c("text_15_cs4k", "text", 15, 11, 4096),
    _c("text_16_cs4k", "text", 16, 11, 4096),
    _c("text_17_cs4k", "text", 17, 11, 4096),
    _c("walk_4095_cs4096", "walk", 4095, 12, 4096),
    _c("walk_4097_cs4096", "walk", 4097, 12, 4096),
    _c("text_40k_pre16k", "text", 40000, 13, 4096, prelearn=16384),
]
