"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference measures on enwik8/enwik9/silesia and similar corpora, none of
which is available here; these generators stand in for them:

* text   -- order-2 Markov chain over the 95 printable ASCII bytes plus
            '\\n'; every (prev2, prev1) row drawn from Dirichlet(alpha=0.1);
            a space is forced after a geometric(p=0.18) word length.  The
            transition rows (the "language") are fixed by seed 0; each text
            segment samples its own path through them.
* walk   -- little-endian int32 random walk, x0 = 0, steps round(N(0, 100^2)).
* random -- uniform bytes (incompressible).
* runs   -- runs of a uniform byte value with geometric lengths of mean 200.

Config builders follow the workload descriptions the benchmark uses:
config0 (1 MiB text, 64 KiB chunks), config1 (256 MiB mixed, 1 MiB chunks,
64 KiB blocks in seeded order), config2 (4096 buffers, log-uniform sizes in
[4 KiB, 4 MiB], one content type each, 256 KiB chunks) and config4 (a
serving request stream: Poisson arrivals, sizes log-uniform in [1 KiB,
16 MiB], 70% compress / 30% decompress, content drawn as in config2).
"""
import concurrent.futures as _cf
import ctypes
import functools
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
_SYMS = np.array(list(range(0x20, 0x7F)) + [0x0A], dtype=np.uint8)  # 96 symbols
_SPACE = 0  # index of 0x20
KINDS = ("text", "walk", "random", "runs")


@functools.lru_cache(maxsize=1)
def _lib():
    path = os.path.join(_PKG, "libcucm_workload.so")
    if not os.path.exists(path):
        from . import build as _b
        _b.build()
    lib = ctypes.CDLL(path)
    lib.wl_markov_text.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64]
    lib.wl_markov_text.restype = None
    return lib


@functools.lru_cache(maxsize=4)
def _language(seed=0):
    k = len(_SYMS)
    rng = np.random.default_rng(seed)
    rows = rng.dirichlet(np.full(k, 0.1), size=k * k)
    cdf = np.cumsum(rows, axis=1)
    cdf = cdf / cdf[:, -1:]
    scaled = np.minimum(np.floor(cdf * 4294967296.0), 4294967295).astype(np.uint32)
    scaled[:, -1] = 0xFFFFFFFF
    return np.ascontiguousarray(scaled.reshape(-1))


def text(n, seed, language_seed=0):
    out = np.empty(n, dtype=np.uint8)
    if n == 0:
        return out
    cdf = _language(language_seed)
    _lib().wl_markov_text(cdf.ctypes.data, _SYMS.ctypes.data, len(_SYMS), _SPACE, 0.18,
                          int(seed) & 0xFFFFFFFFFFFFFFFF, out.ctypes.data, n)
    return out


def walk(n, seed):
    rng = np.random.default_rng(seed)
    m = (n + 3) // 4
    steps = np.rint(rng.normal(0.0, 100.0, size=max(m - 1, 0))).astype(np.int64)
    x = np.concatenate([[0], np.cumsum(steps)]).astype(np.int64)
    v = (x & 0xFFFFFFFF).astype(np.uint32).astype("<u4")
    return np.frombuffer(v.tobytes(), dtype=np.uint8)[:n].copy()


def random_bytes(n, seed):
    return np.random.default_rng(seed).integers(0, 256, size=n, dtype=np.uint8)


def runs(n, seed):
    rng = np.random.default_rng(seed)
    parts = [np.empty(0, dtype=np.uint8)]
    total = 0
    while total < n:
        k = max(16, (n - total) // 150 + 16)
        lens = rng.geometric(1.0 / 200.0, size=k)
        vals = rng.integers(0, 256, size=k, dtype=np.uint8)
        parts.append(np.repeat(vals, lens))
        total += int(lens.sum())
    out = np.concatenate(parts)[:n]
    return out.copy()


def make(kind, n, seed):
    if kind == "text":
        return text(n, seed)
    if kind == "walk":
        return walk(n, seed)
    if kind == "random":
        return random_bytes(n, seed)
    if kind == "runs":
        return runs(n, seed)
    raise ValueError(kind)


def _parallel(fn, items):
    """fn over items on host threads (the generators release the GIL in C
    and numpy); results in item order, identical to a serial run."""
    with _cf.ThreadPoolExecutor(max(1, min(32, os.cpu_count() or 1))) as ex:
        return list(ex.map(fn, items))


def _derive(seed, i):
    return int(np.random.SeedSequence([seed, i]).generate_state(1, dtype=np.uint64)[0])


def long_text(total, seed, piece=4 << 20):
    """`total` bytes of the Markov text in `piece`-byte pieces, each its own
    seeded walk of the same language, generated on host threads."""
    out = np.empty(total, dtype=np.uint8)

    def fill(i):
        a = i * piece
        out[a:a + piece] = text(min(piece, total - a), _derive(seed, i))

    _parallel(fill, range((total + piece - 1) // piece))
    return out


def config0():
    """1 MiB of Markov text; 64 KiB chunks (16 chunks)."""
    return text(1 << 20, _derive(0, 0)), dict(chunksize=64 << 10, unit=128, prelearn=0, batch=100)


def config1(total=256 << 20, block=64 << 10):
    """Mixed buffer of `total` bytes in 64 KiB blocks: 50% text, 25% int32
    walk, 15% random, 10% runs, in seeded order; 1 MiB chunks."""
    nblocks = total // block
    counts = [int(round(nblocks * f)) for f in (0.5, 0.25, 0.15, 0.10)]
    counts[0] += nblocks - sum(counts)
    kinds = np.repeat(np.arange(4), counts)
    rng = np.random.default_rng(1)
    rng.shuffle(kinds)
    out = np.empty(nblocks * block, dtype=np.uint8)

    def fill(i):
        out[i * block:(i + 1) * block] = make(KINDS[kinds[i]], block, _derive(1, i))

    _parallel(fill, range(nblocks))
    return out, dict(chunksize=1 << 20, unit=128, prelearn=0, batch=100)


def config2_sizes(count=4096, lo=4096, hi=4 << 20, seed=2):
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))).astype(np.int64)
    kinds = rng.choice(4, size=count, p=[0.5, 0.25, 0.15, 0.10])
    return sizes, kinds


def config2(count=4096, lo=4096, hi=4 << 20, seed=2):
    """`count` independent buffers with log-uniform sizes in [lo, hi], one
    content type each (0.5 text / 0.25 walk / 0.15 random / 0.1 runs);
    256 KiB chunks."""
    sizes, kinds = config2_sizes(count, lo, hi, seed)
    bufs = _parallel(lambda i: make(KINDS[kinds[i]], int(sizes[i]), _derive(seed, 1000 + i)), range(count))
    return bufs, dict(chunksize=256 << 10, unit=128, prelearn=0, batch=100)


def config2_sample(k=512, count=4096):
    """A stratified sample of config2's buffers: every (count / k)-th buffer
    in size order, the largest included.  Sorted buffer indices."""
    sizes, _ = config2_sizes(count)
    order = sorted(range(count), key=lambda i: (int(sizes[i]), i))
    step = max(1, count // k)
    pick = order[::step][:k]
    if order[-1] not in pick:
        pick[-1] = order[-1]
    return sorted(pick)


def config4(count, offered_gbps, lo=1024, hi=16 << 20, seed=4):
    """A serving request stream of `count` requests at an offered load of
    `offered_gbps` GB/s: Poisson arrivals (exponential gaps whose mean is the
    mean request size over the load), sizes log-uniform in [lo, hi], 70%
    compress / 30% decompress, content drawn as in config2; 256 KiB chunks.
    Returns (arrival seconds, is_compress flags, buffers, params)."""
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))).astype(np.int64)
    kinds = rng.choice(4, size=count, p=[0.5, 0.25, 0.15, 0.10])
    comp = rng.random(count) < 0.7
    mean = (hi - lo) / np.log(hi / lo)
    gaps = rng.exponential(mean / (offered_gbps * 1e9), size=count)
    arrivals = np.cumsum(gaps) - gaps[0]
    bufs = [make(KINDS[k], int(s), _derive(seed, 5000 + i)) for i, (s, k) in enumerate(zip(sizes, kinds))]
    return arrivals, comp, bufs, dict(chunksize=256 << 10, unit=128, prelearn=0, batch=100)
