#!/usr/bin/env python3
"""SHA-256 manifest of the reference's containers for the full-size workloads.

The reference ships no test vectors, so these digests come from running the
reference itself: oracle/_ref/cucm_compress_ref, its unmodified sources built
for the host by oracle/make_ref.py (run `make -C oracle ref` first, in a
checkout that has the reference sources).  Only digests are committed, not
the containers (hundreds of MB).

* mixed256M -- the 256 MiB mixed buffer (workloads.config1), 1 MiB chunks,
  unit 128, batch 100: 256 chunks.  The reference codes every chunk of a
  stream from the zero model with zero history before the chunk start, and a
  chunk's payload does not depend on the batch it sits in, so each 1 MiB
  chunk is compressed by the reference as a file of its own (one process per
  chunk, all host cores) and the payloads are framed into the 256-chunk
  container exactly as the reference's writer frames them
  (cucm_compress_v2.cu:1197-1244: 21-byte big-endian header, then per batch
  of <= 100 chunks a little-endian u32 body size, big-endian u32 inclusive
  end offsets from the body start, and the payloads).  The framing itself is
  pinned by the small golden containers (batches 1/2/3/100).
* many4096 -- the 4096 buffers of workloads.config2 (log-uniform 4 KiB ..
  4 MiB, 256 KiB chunks, unit 128, batch 100): each buffer is its own
  container, written by the reference's CLI directly.  The digest of every
  container is kept, with its length.

Usage:  python tests/golden/make_fullsize.py [--only mixed256M|many4096] [--jobs N]
"""
import argparse
import concurrent.futures as cf
import hashlib
import json
import os
import struct
import subprocess
import sys
import tempfile
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cucm_b200 import workloads as W  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "cucm_compress_ref")
OUT = os.path.join(HERE, "fullsize_manifest.json")
HEADER = 21
# Host memory the reference's compressor holds per chunk of a batch: eight
# 2^25-slot state arrays plus their probability tables.
BYTES_PER_CHUNK = 8 * ((1 << 25) + 1024)


def sha(b):
    return hashlib.sha256(b).hexdigest()


def run_ref(src, dst, chunksize, unit=128, batch=100):
    subprocess.run([REF, "-f", src, "-o", dst, "-s", str(chunksize), "-u", str(unit), "-b", str(batch)],
                   check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    with open(dst, "rb") as f:
        return f.read()


class MemGate:
    """Admits jobs while their summed host-memory estimate fits a budget."""

    def __init__(self, budget):
        self.budget, self.used = budget, 0
        self.cv = threading.Condition()

    def __enter__(self):
        return self

    def take(self, n):
        n = min(n, self.budget)
        with self.cv:
            while self.used + n > self.budget:
                self.cv.wait()
            self.used += n
        return n

    def give(self, n):
        with self.cv:
            self.used -= n
            self.cv.notify_all()

    def __exit__(self, *a):
        return False


def frame(orig_size, chunksize, unit, batch, payloads):
    """The reference's container around per-chunk payloads (no prelearn)."""
    out = bytearray(struct.pack(">IHHIIIB", orig_size, batch, unit, chunksize, 0, 0, 0))
    for b0 in range(0, len(payloads), batch):
        group = payloads[b0:b0 + batch]
        c = len(group)
        ends, pos = [], 4 * c - 1
        for p in group:
            pos += len(p)
            ends.append(pos)
        body = b"".join(struct.pack(">I", e) for e in ends) + b"".join(group)
        out += struct.pack("<I", len(body)) + body
    return bytes(out)


def mixed256m(jobs):
    data, p = W.config1()
    cs = p["chunksize"]
    n = data.size
    nchunks = n // cs
    t0 = time.time()
    with tempfile.TemporaryDirectory() as tmp:
        def one(i):
            src = os.path.join(tmp, "c%d.bin" % i)
            dst = src + ".cucm"
            with open(src, "wb") as f:
                f.write(data[i * cs:(i + 1) * cs].tobytes())
            blob = run_ref(src, dst, cs, p["unit"], p["batch"])
            os.remove(src)
            os.remove(dst)
            (body,) = struct.unpack("<I", blob[HEADER:HEADER + 4])
            (end,) = struct.unpack(">I", blob[HEADER + 4:HEADER + 8])
            assert len(blob) == HEADER + 4 + body and end == body - 1, "unexpected one-chunk container"
            return blob[HEADER + 8:]
        with cf.ThreadPoolExecutor(jobs) as ex:
            payloads = list(ex.map(one, range(nchunks)))
    blob = frame(n, cs, p["unit"], p["batch"], payloads)
    print("mixed256M: %d chunks in %.0f s -> %d bytes" % (nchunks, time.time() - t0, len(blob)))
    return {"workload": "workloads.config1(): 256 MiB mixed, 1 MiB chunks, unit 128, batch 100",
            "input_sha256": sha(data.tobytes()), "input_len": int(n), "chunks": nchunks,
            "output_sha256": sha(blob), "output_len": len(blob),
            "chunk_payload_lens": [len(x) for x in payloads]}


def many4096(jobs, mem_budget):
    bufs, p = W.config2()
    cs = p["chunksize"]
    gate = MemGate(mem_budget)
    order = sorted(range(len(bufs)), key=lambda i: -len(bufs[i]))  # longest first
    digests, lens = [None] * len(bufs), [None] * len(bufs)
    t0 = time.time()
    done = [0]
    lock = threading.Lock()
    with tempfile.TemporaryDirectory() as tmp:
        def one(i):
            b = bufs[i]
            chunks = max(1, (len(b) + cs - 1) // cs)
            held = gate.take(chunks * BYTES_PER_CHUNK + (64 << 20))
            try:
                src = os.path.join(tmp, "b%d.bin" % i)
                dst = src + ".cucm"
                with open(src, "wb") as f:
                    f.write(b.tobytes())
                blob = run_ref(src, dst, cs, p["unit"], p["batch"])
                os.remove(src)
                os.remove(dst)
            finally:
                gate.give(held)
            digests[i], lens[i] = sha(blob), len(blob)
            with lock:
                done[0] += 1
                if done[0] % 256 == 0:
                    print("many4096: %d / %d buffers, %.0f s" % (done[0], len(bufs), time.time() - t0), flush=True)
        with cf.ThreadPoolExecutor(jobs) as ex:
            list(ex.map(one, order))
    h = hashlib.sha256()
    for b in bufs:
        h.update(struct.pack("<Q", len(b)))
        h.update(b.tobytes())
    print("many4096: %d buffers in %.0f s" % (len(bufs), time.time() - t0))
    return {"workload": "workloads.config2(): 4096 buffers, log-uniform 4 KiB..4 MiB, 256 KiB chunks, unit 128, "
                        "batch 100; one container per buffer",
            "inputs_sha256": h.hexdigest(), "input_lens": [len(b) for b in bufs],
            "output_sha256": digests, "output_len": lens}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["mixed256M", "many4096"])
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--mem-gb", type=float, default=40.0, help="host memory the reference processes may hold")
    a = ap.parse_args()
    if not os.path.exists(REF):
        sys.exit("reference binary missing; run `make -C oracle ref`")
    man = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            man = json.load(f)
    if a.only in (None, "mixed256M"):
        man["mixed256M"] = mixed256m(a.jobs)
        with open(OUT, "w") as f:
            json.dump(man, f, separators=(",", ":"))
    if a.only in (None, "many4096"):
        man["many4096"] = many4096(a.jobs, int(a.mem_gb * (1 << 30)))
        with open(OUT, "w") as f:
            json.dump(man, f, separators=(",", ":"))


if __name__ == "__main__":
    main()
