#!/usr/bin/env python3
"""Benchmark of the CuCM coder on the 256 MiB mixed workload at 1 MiB chunks.

Workload (one "step"): compress the 256 MiB mixed buffer (50% Markov text,
25% int32 walk, 15% random, 10% runs in 64 KiB blocks; 1 MiB chunks,
unit 128, no prelearn, batch 100 -- 256 chunks) and decompress the result
back, byte-exact.  `value` is the round trip in MB/s of uncompressed bytes
(input bytes / (compress time + decompress time)), whole job over all ranks,
with the buffers resident in HBM; compress and decompress are also reported
alone.  The input (256 MiB, plus 48 GiB of chunk tables touched at random)
is larger than L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload mixed256M|batch|serve|small]

The headline line also carries, unless --no-extras: "batched_vs_plain" (the
4096-buffer set, batched persistent form against the plain form on a
stratified 512-buffer sample, every batched container hashed against the
reference's) and "serve" (the serving loop at offered loads of 2, 8 and
32 GB/s, 32 requests each, p50/p99 latency and sustained MB/s against one
request at a time).  "sha256_match" compares the timed workload's container
with the reference's.

Other workloads (one JSON line each, not the headline):
  batch  -- 4096 independent buffers, log-uniform 4 KiB..4 MiB, 256 KiB chunks:
            the batched persistent form (one launch for all buffers) against
            the plain form (one launch per chunk), byte-identical outputs;
  serve  -- the serving loop under Poisson request streams at stated offered
            loads: p50/p99 latency and sustained MB/s against serving the
            same stream one request at a time;
  small  -- 1 MiB of text at 64 KiB chunks, one round trip (profiling case).

--impl reference times the reference's own implementation of the path on the
host cores: its two programs built for the CPU from its unmodified sources
(oracle/_ref), one chunk per process on all cores, on a bounded sample of
the same workload.  Under torchrun, rank 0 alone runs it.

Multi-GPU (--gpus N; started under torchrun by the script itself when run
alone): one process per GPU, one stream of N x 256 MiB split into
contiguous chunk ranges, one per rank (cucm_b200/sharded.py).  The chunk
bodies are gathered to rank 0 and framed into one container; rank 0
broadcasts it, every rank decodes its range and the bytes go back to rank 0.
Weak scaling; the slowest rank's time is used.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ALGO_BYTES_PER_BYTE = 4096  # 8 bits x 8 orders x (32 B sector gather + 32 B write-back)
PARAMS = dict(chunksize=1 << 20, unit=128, prelearn=0, batch=100)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="persistent", choices=["persistent", "plain"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="mixed256M", choices=["mixed256M", "batch", "serve", "small", "fixed"])
    ap.add_argument("--autotune", action="store_true",
                    help="mixed256M: choose the execution form with the measured autotuner first (untimed, on a "
                         "32 MiB sample cut into the same 256 chunks)")
    ap.add_argument("--plain-sample", type=int, default=512, help="buffers the plain form codes (batch)")
    ap.add_argument("--requests", type=int, default=48, help="requests per offered load (serve)")
    ap.add_argument("--no-extras", action="store_true",
                    help="mixed256M: leave out the batched-vs-plain and serving figures of the headline line")
    ap.add_argument("--extra-requests", type=int, default=32,
                    help="requests per offered load of the headline line's serving figures")
    ap.add_argument("--loads", default="0.02,0.2,2,8,32", help="offered loads in GB/s (serve)")
    ap.add_argument("--small-bytes", type=int, default=1 << 20, help="bytes of the small workload")
    ap.add_argument("--small-source", default="text", choices=["text", "mixed"],
                    help="small workload content: text, or the head of the 256 MiB mixed buffer")
    ap.add_argument("--small-chunk", type=int, default=64 << 10, help="chunk size of the small workload")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def reduce_max(vals, dist=None, device="cpu"):
    """Element-wise max over ranks of per-rank figures (the slowest rank's
    device times); the identity without a process group."""
    if dist is None:
        return [float(v) for v in vals]
    import torch
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def reference_sha256(key):
    """SHA-256 of the reference's container for a full-size workload, from the
    committed manifest (tests/golden/fullsize_manifest.json, written by the
    reference's own compressor), or None."""
    p = os.path.join(ROOT, "tests", "golden", "fullsize_manifest.json")
    try:
        with open(p) as f:
            return json.load(f)[key]["output_sha256"]
    except Exception:
        return None


def profile_traffic():
    """DRAM bytes per full-size launch of each kernel, from the committed ncu
    summary (profiles/traffic_mixed256M.json), if present."""
    p = os.path.join(ROOT, "profiles", "traffic_mixed256M.json")
    try:
        with open(p) as f:
            return {k: v.get("dram_bytes_per_launch") for k, v in json.load(f).items() if isinstance(v, dict)}
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
             "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU runs of the reference's own code (oracle/_ref) on a bounded sample.

def _ref_bins():
    c = os.path.join(ROOT, "oracle", "_ref", "cucm_compress_ref")
    d = os.path.join(ROOT, "oracle", "_ref", "cucm_decompress_ref")
    if os.path.exists(c) and os.path.exists(d):
        return c, d, "reference"
    cli = os.path.join(ROOT, "oracle", "oracle_cli")
    if not os.path.exists(cli):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle_cli"], check=True)
    return cli, cli, "port"


def _host_procs():
    n = os.cpu_count() or 1
    try:
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable"):
                    gb = int(ln.split()[1]) / (1 << 20)
                    n = min(n, max(1, int(gb / 1.2)))
    except Exception:
        pass
    return max(1, min(n, 64))


def cpu_round_trip(data, nchunks, tmp):
    """Compress then decompress `nchunks` 1 MiB chunks of `data`, one process
    per chunk, all at once.  Returns (compress_s, decompress_s, kind)."""
    comp, decomp, kind = _ref_bins()
    cs = PARAMS["chunksize"]
    files = []
    for i in range(nchunks):
        p = os.path.join(tmp, "c%d.bin" % i)
        with open(p, "wb") as f:
            f.write(data[i * cs:(i + 1) * cs].tobytes())
        files.append(p)

    def run_all(cmds):
        t = time.perf_counter()
        procs = [subprocess.Popen(c, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL) for c in cmds]
        rcs = [p.wait() for p in procs]
        if any(rcs):
            raise RuntimeError("CPU baseline run failed: %s" % rcs)
        return time.perf_counter() - t

    if kind == "reference":
        cc = [[comp, "-f", f, "-o", f + ".cucm", "-s", str(cs), "-u", "128", "-b", "100"] for f in files]
        dd = [[decomp, "-i", f + ".cucm", "-o", f + ".out"] for f in files]
    else:
        cc = [[comp, "c", f, f + ".cucm", str(cs), "128", "0", "100", "1"] for f in files]
        dd = [[decomp, "d", f + ".cucm", f + ".out", "1"] for f in files]
    tc = run_all(cc)
    td = run_all(dd)
    for f in files:
        with open(f, "rb") as a, open(f + ".out", "rb") as b:
            if a.read() != b.read():
                raise RuntimeError("CPU baseline round trip mismatch")
    return tc, td, kind


def cpu_baseline(data):
    n = _host_procs()
    with tempfile.TemporaryDirectory() as tmp:
        tc, td, kind = cpu_round_trip(data, n, tmp)
    mb = n * PARAMS["chunksize"] / 1e6
    return {"value": mb / (tc + td), "unit": "MB/s", "cores": n, "kind": kind,
            "sample": "%d of the 256 chunks (1 MiB each), one process per chunk, compress then decompress" % n,
            "compress_MBps": mb / tc, "decompress_MBps": mb / td}


# ---------------------------------------------------------------------------

def headline_config():
    """The headline workload, the same in both arms (the CPU arm's sample of
    it is described in its cpu_baseline)."""
    return {"workload": "mixed 256 MiB per rank, 1 MiB chunks (256), unit 128, batch 100",
            "chunksize": PARAMS["chunksize"], "unit": PARAMS["unit"], "batch": PARAMS["batch"],
            "parallelism": "independent chunks per rank", "l2": "inputs larger than L2"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from cucm_b200 import workloads as W
    data, _ = W.config1()
    n = _host_procs()
    times = []
    with tempfile.TemporaryDirectory() as tmp:
        for step in range(args.warmup + args.steps):
            tc, td, kind = cpu_round_trip(data, n, tmp)
            if step >= args.warmup:
                times.append((tc, td))
    tc = sum(t[0] for t in times)
    td = sum(t[1] for t in times)
    mb = n * PARAMS["chunksize"] / 1e6 * len(times)
    value = mb / (tc + td)
    line = {
        "impl": "reference", "metric": "compress+decompress round-trip MB/s", "value": value, "unit": "MB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * (tc + td) / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": headline_config(),
        "compress_MBps": mb / tc, "decompress_MBps": mb / td,
        "cpu_baseline": {"value": value, "unit": "MB/s", "cores": n, "kind": kind,
                         "sample": "%d of the 256 chunks (1 MiB each) per step, one process per chunk, "
                                   "compress then decompress" % n},
        "e2e": {"value": value, "unit": "MB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def relaunch_under_torchrun(args):
    """`--gpus N` outside torchrun: start the N ranks (one per GPU) by
    running this script again under torch.distributed.run on this node."""
    import socket
    with socket.socket() as s_:
        s_.bind(("127.0.0.1", 0))
        port = s_.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=%d" % args.gpus,
           "--master-addr=127.0.0.1", "--master-port=%d" % port, os.path.abspath(__file__)] + sys.argv[1:]
    os.execv(sys.executable, cmd)


def run_sharded(args, rank, world, local):
    """N GPUs, one rank each: one stream of N x 256 MiB whose N blocks are
    the 256 MiB mixed buffer, 1 MiB chunks.  Each rank owns a contiguous range
    of 256 chunks.  Compress: every rank codes its range, the body sizes are
    all-gathered and the bodies sent to rank 0 (NCCL), which frames the
    container.  Decompress: rank 0 broadcasts the container, every rank
    decodes its range and sends it back.  Weak scaling; each phase is timed
    with CUDA events (exchanges included), synchronised on both sides, and
    the slowest rank's time is used."""
    import datetime
    import torch
    import torch.distributed as dist
    import cucm_b200 as cc
    from cucm_b200 import sharded
    from cucm_b200 import workloads as W
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    data, _ = W.config1()
    n = data.size
    total = n * world
    cs, unit, batch = PARAMS["chunksize"], PARAMS["unit"], PARAMS["batch"]
    assert sharded.split_chunks(total // cs, world)[rank] == (rank * (n // cs), n // cs)
    ctx = cc.Context(local)
    coder = sharded.DeviceCoder(ctx, dev)
    d_in = torch.from_numpy(data).to(dev)
    h_in = torch.from_numpy(data).pin_memory()
    h_out = torch.empty(total, dtype=torch.uint8).pin_memory() if rank == 0 else None

    def step(host):
        torch.cuda.synchronize()
        dist.barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record()
        block = d_in
        if host:
            block = torch.empty_like(d_in)
            block.copy_(h_in, non_blocking=True)
            torch.cuda.current_stream().synchronize()
        cont = sharded.compress_sharded(coder, block, total, cs, unit, batch, dist=dist)
        ev[1].record()
        back = sharded.decompress_sharded(coder, cont, total, cs, dist=dist)
        if host and rank == 0:
            h_out.copy_(back, non_blocking=True)
        ev[2].record()
        torch.cuda.synchronize()
        return cont, back, ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])

    ok = True
    cont = None
    for _ in range(max(args.warmup, 1)):
        cont, back, _, _ = step(False)
        if rank == 0:
            ok = ok and all(torch.equal(back[r * n:(r + 1) * n], d_in) for r in range(world))
    comp_n = cont.numel() if rank == 0 else 0
    sampler = ClockSampler(local)
    sampler.start()
    tc = td = 0.0
    for _ in range(args.steps):
        _, _, a, b = step(False)
        tc += a
        td += b
    clocks = sampler.stop()
    t_all, t_c, t_d = reduce_max([tc + td, tc, td], dist, dev)
    e_ms = 0.0
    for i in range(args.steps + 1):
        _, _, a, b = step(True)
        if i:
            e_ms += a + b
    if rank == 0:
        ok = ok and all(torch.equal(h_out[r * n:(r + 1) * n], h_in) for r in range(world))
    e_max = reduce_max([e_ms], dist, dev)[0]
    K = max(args.steps, 1)
    if rank == 0:
        line = {
            "metric": "compress+decompress round-trip MB/s", "value": total * K / (t_all / 1e3) / 1e6,
            "unit": "MB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_all / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8", "data": "synthetic",
            "config": {"workload": "one stream of %d x 256 MiB (the mixed buffer per rank), 1 MiB chunks, unit 128, "
                                   "batch 100" % world, "chunksize": cs, "unit": unit, "batch": batch,
                       "parallelism": "contiguous chunk ranges per rank; bodies gathered and framed on rank 0, "
                                      "container broadcast, ranges decoded per rank and gathered (NCCL)",
                       "l2": "inputs larger than L2"},
            "compress_MBps": total * K / (t_c / 1e3) / 1e6, "decompress_MBps": total * K / (t_d / 1e3) / 1e6,
            "compressed_bytes": int(comp_n), "byte_exact": bool(ok),
            "e2e": {"value": total * K / (e_max / 1e3) / 1e6, "unit": "MB/s", "h2d_bytes_per_step": total,
                    "d2h_bytes_per_step": total},
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()
    if not ok:
        raise SystemExit("sharded round trip mismatch")


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        relaunch_under_torchrun(args)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload != "mixed256M":
        if rank == 0:
            {"batch": run_batch, "serve": run_serve, "small": run_small, "fixed": run_fixed}[args.workload](args)
        return
    if world > 1:
        run_sharded(args, rank, world, local)
        return
    import numpy as np
    import torch
    import cucm_b200 as cc
    from cucm_b200 import workloads as W

    dist = None  # the single-GPU path; N > 1 runs run_sharded
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    data, _ = W.config1()
    n = data.size
    form = cc.FORM_PLAIN if args.form == "plain" else cc.FORM_PERSISTENT
    ctx = cc.Context(local, form=form)
    tuned = None
    if args.autotune:
        nch = n // PARAMS["chunksize"]
        sample = data[:32 << 20]
        best, cands = ctx.autotune(sample, reps=1, chunksize=max(sample.size // max(nch, 1), 4096),
                                   unit=PARAMS["unit"], batch=PARAMS["batch"])
        keys = ("form", "kernel", "cmp_ctas", "dec_pairs", "dec_tables")
        tuned = {"chosen": {k: best[k] for k in keys},
                 "sample": "first 32 MiB, %d chunks" % nch,
                 "candidates": [{k: c[k] for k in keys + ("compress_ms", "decompress_ms")} for c in cands]}
    p = cc.default_params(**PARAMS)
    cap = cc.lib().cucm_compress_bound(n, p)
    d_in = torch.from_numpy(data).to(dev)
    d_comp = torch.empty(cap, dtype=torch.uint8, device=dev)
    d_dec = torch.empty(n, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()

    def step():
        m = ctx.compress_dev(d_in.data_ptr(), n, d_comp.data_ptr(), cap, **PARAMS)
        sc = ctx.last_stats()
        ctx.decompress_dev(d_comp.data_ptr(), m, d_dec.data_ptr(), n)
        sd = ctx.last_stats()
        return m, sc, sd

    for _ in range(max(args.warmup, 0)):
        comp_n, _, _ = step()
    if not torch.equal(d_dec, d_in):
        raise SystemExit("round trip mismatch on the device")
    # the container of the timed workload against the reference's (by hash)
    import hashlib
    got_sha = hashlib.sha256(d_comp[:comp_n].cpu().numpy().tobytes()).hexdigest() if args.warmup > 0 else None
    want_sha = reference_sha256("mixed256M")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    tc = td = kc = kd = 0.0
    launches = 0
    for _ in range(args.steps):
        comp_n, sc, sd = step()
        tc += sc["device_ms"]
        td += sd["device_ms"]
        kc += sc["kernel_ms"]
        kd += sd["kernel_ms"]
        launches += sc["launches"] + sd["launches"]
    barrier()
    clocks = sampler.stop()
    t_all, t_c, t_d = reduce_max([tc + td, tc, td], dist, dev)
    K = max(args.steps, 1)
    total_bytes = world * n * K
    value = total_bytes / (t_all / 1e3) / 1e6

    # End to end through the host-buffer API: pinned host input, host output.
    e2e = None
    if not args.no_e2e:
        h_in = torch.from_numpy(data).pin_memory()
        ptr = h_in.data_ptr()
        import ctypes
        h_out = torch.empty(cap, dtype=torch.uint8).pin_memory()
        h_back = torch.empty(n, dtype=torch.uint8).pin_memory()
        got = ctypes.c_uint64()
        e_ms = 0.0
        h2d = d2h = 0
        for i in range(K + 1):
            rc = cc.lib().cucm_compress(ctx._h, ptr, n, p, h_out.data_ptr(), cap, ctypes.byref(got))
            if rc:
                raise cc.CucmError(rc, "cucm_compress")
            ms1 = ctx.last_stats()["device_ms"]
            m = got.value
            rc = cc.lib().cucm_decompress(ctx._h, h_out.data_ptr(), m, h_back.data_ptr(), n, ctypes.byref(got))
            if rc:
                raise cc.CucmError(rc, "cucm_decompress")
            ms2 = ctx.last_stats()["device_ms"]
            if i > 0:  # first pass warms the host-buffer path
                e_ms += ms1 + ms2
                h2d += n + m
                d2h += m + n
        if not torch.equal(h_back, h_in):
            raise SystemExit("host round trip mismatch")
        e_max = reduce_max([e_ms], dist, dev)[0]
        e2e = {"value": world * n * K / (e_max / 1e3) / 1e6, "unit": "MB/s",
               "h2d_bytes_per_step": h2d // K, "d2h_bytes_per_step": d2h // K}

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    peak, peak_kind = measured_peak()
    traffic = profile_traffic()

    def roof(kernel, ms_per_launch):
        ach = ALGO_BYTES_PER_BYTE * n / (ms_per_launch / 1e3) / 1e9 if ms_per_launch > 0 else None
        return {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": (ach / peak) if ach else None, "traffic": traffic.get(kernel) if traffic else None,
                "peak_source": peak_kind, "kernel": kernel, "algorithmic_bytes_per_launch": ALGO_BYTES_PER_BYTE * n,
                "kernel_ms_per_launch": ms_per_launch}
    r_comp = roof("compress_fast_kernel", kc / K)
    r_dec = roof("decompress_pair_kernel", kd / K)
    # the dominant kernel of the step (the longer one) carries the roofline
    roofline = dict(r_dec if kd >= kc else r_comp)
    roofline["other"] = r_comp if kd >= kc else r_dec
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(data)
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "error": str(e)}
    line = {
        "metric": "compress+decompress round-trip MB/s", "value": value, "unit": "MB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_all / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": headline_config(),
        "execution": {"form": args.form, "tuning": ctx.get_tuning()},
        "compress_MBps": world * n * K / (t_c / 1e3) / 1e6, "decompress_MBps": world * n * K / (t_d / 1e3) / 1e6,
        "compressed_bytes": int(comp_n), "ratio": n / comp_n,
        "sha256_match": (got_sha == want_sha) if (got_sha and want_sha) else None,
        "sha256_reference": "container of the reference's own compressor (tests/golden/fullsize_manifest.json)",
        "kernel_ms": {"compress": kc / K, "decompress": kd / K},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
        "gpu_launches": launches,
    }
    if tuned:
        line["autotune"] = tuned
    if world == 1 and not args.no_extras:
        # configs 2-4 beside the headline: the device is handed over whole
        ctx.close()
        del d_in, d_comp, d_dec
        torch.cuda.empty_cache()
        line["plain_form"] = plain_measure(data)
        torch.cuda.empty_cache()
        line["batched_vs_plain"] = batch_measure(warmup=1, sample=512)
        torch.cuda.empty_cache()
        line["serve"] = serve_measure([2.0, 8.0, 32.0], args.extra_requests)
        torch.cuda.empty_cache()
        line["fixed_model"] = fixed_measure()
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Other workloads

def _mbps(nbytes, ms):
    return nbytes / (ms / 1e3) / 1e6 if ms > 0 else None


def run_small(args):
    """A small case of the same path -- by default 1 MiB of text at 64 KiB
    chunks, or the head of the 256 MiB mixed buffer -- one compress and one
    decompress through the device API: the case the ncu captures use."""
    import torch
    import cucm_b200 as cc
    from cucm_b200 import workloads as W
    if args.small_source == "text":
        data, _ = W.config0()
    else:
        data, _ = W.config1()
    data = data[:args.small_bytes].copy()
    p = dict(PARAMS, chunksize=args.small_chunk)
    n = data.size
    ctx = cc.Context(0)
    d_in = torch.from_numpy(data).cuda()
    cap = cc.lib().cucm_compress_bound(n, cc.default_params(**p))
    d_c = torch.empty(cap, dtype=torch.uint8, device="cuda")
    d_o = torch.empty(n, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    m = ctx.compress_dev(d_in.data_ptr(), n, d_c.data_ptr(), cap, **p)
    sc = ctx.last_stats()
    ctx.decompress_dev(d_c.data_ptr(), m, d_o.data_ptr(), n)
    sd = ctx.last_stats()
    ok = bool(torch.equal(d_o, d_in))
    print(json.dumps({"metric": "small round trip MB/s",
                      "workload": "%d bytes of %s, %d-byte chunks (%d)" % (n, args.small_source, p["chunksize"],
                                                                         (n + p["chunksize"] - 1) // p["chunksize"]),
                      "compress_MBps": _mbps(n, sc["device_ms"]), "decompress_MBps": _mbps(n, sd["device_ms"]),
                      "kernel_ms": {"compress": sc["kernel_ms"], "decompress": sd["kernel_ms"]},
                      "compressed_bytes": m, "byte_exact": ok}), flush=True)
    if not ok:
        raise SystemExit("round trip mismatch")


def plain_measure(data, reps=1):
    """The headline buffer (256 MiB mixed, 1 MiB chunks) in the plain form:
    one single-CTA kernel launch per chunk, on up to 128 streams, as the
    reference launches per chunk; one untimed warm-up, then `reps` round
    trips, device time per call; the container is hashed against the
    reference's."""
    import hashlib
    import torch
    import cucm_b200 as cc
    n = data.size
    ctx = cc.Context(0, form=cc.FORM_PLAIN)
    cap = cc.lib().cucm_compress_bound(n, cc.default_params(**PARAMS))
    d_in = torch.from_numpy(data).cuda()
    d_c = torch.empty(cap, dtype=torch.uint8, device="cuda")
    d_o = torch.empty(n, dtype=torch.uint8, device="cuda")
    tc = td = 0.0
    launches = 0
    for i in range(reps + 1):
        m = ctx.compress_dev(d_in.data_ptr(), n, d_c.data_ptr(), cap, **PARAMS)
        sc = ctx.last_stats()
        ctx.decompress_dev(d_c.data_ptr(), m, d_o.data_ptr(), n)
        sd = ctx.last_stats()
        if i:
            tc += sc["kernel_ms"]
            td += sd["kernel_ms"]
            launches = sc["launches"] + sd["launches"]
    ok = bool(torch.equal(d_o, d_in))
    got = hashlib.sha256(d_c[:m].cpu().numpy().tobytes()).hexdigest()
    want = reference_sha256("mixed256M")
    ctx.close()
    del d_in, d_c, d_o
    return {"workload": "the headline buffer, plain form: one single-CTA launch per chunk on up to 128 streams",
            "compress_MBps": _mbps(n * reps, tc), "decompress_MBps": _mbps(n * reps, td),
            "round_trip_MBps": _mbps(n * reps, tc + td),
            "kernel_ms": {"compress": tc / reps, "decompress": td / reps}, "launches_per_round_trip": launches,
            "sha256_match": (got == want) if want else None, "byte_exact": ok}


def batch_measure(warmup=1, sample=512):
    """Configs 2 / 3: the 4096 buffers, batched persistent form (one launch
    for every chunk of every buffer) against the plain form (one launch per
    chunk) on a stratified sample of `sample` buffers (every n/k-th buffer in
    size order, smallest and largest included), device buffers, plus every
    batched container hashed against the reference's."""
    import hashlib
    import torch
    import cucm_b200 as cc
    from cucm_b200 import workloads as W
    bufs, p = W.config2()
    cs = p["chunksize"]
    ctx = cc.Context(0)

    def dev_round(sub, form):
        ctx.set_tuning(form=form)
        d_in = [torch.from_numpy(b).cuda() if len(b) else torch.zeros(1, dtype=torch.uint8, device="cuda")
                for b in sub]
        caps = [cc.many_cap(len(b), cs) for b in sub]
        d_out = [torch.empty(c, dtype=torch.uint8, device="cuda") for c in caps]
        back = [torch.empty(max(len(b), 1), dtype=torch.uint8, device="cuda") for b in sub]
        torch.cuda.synchronize()
        sizes, st = ctx.compress_many_dev([(x.data_ptr(), len(b)) for x, b in zip(d_in, sub)],
                                          [(x.data_ptr(), c) for x, c in zip(d_out, caps)], **p)
        sc = ctx.last_stats()
        if any(st):
            raise SystemExit("compress_many_dev failed: %s" % sorted(set(st)))
        _, st2 = ctx.decompress_many_dev([(x.data_ptr(), m) for x, m in zip(d_out, sizes)],
                                         [(x.data_ptr(), len(b)) for x, b in zip(back, sub)])
        sd = ctx.last_stats()
        if any(st2):
            raise SystemExit("decompress_many_dev failed: %s" % sorted(set(st2)))
        ok = all(torch.equal(x[:len(b)], y[:len(b)]) for x, y, b in zip(back, d_in, sub))
        digests = [hashlib.sha256(x[:m].cpu().numpy().tobytes()).hexdigest() for x, m in zip(d_out, sizes)]
        nb = sum(len(b) for b in sub)
        del d_in, d_out, back
        return dict(buffers=len(sub), bytes=nb, compressed=sum(sizes), compress_ms=sc["device_ms"],
                    decompress_ms=sd["device_ms"], compress_launches=sc["launches"],
                    decompress_launches=sd["launches"], compress_MBps=_mbps(nb, sc["device_ms"]),
                    decompress_MBps=_mbps(nb, sd["device_ms"]),
                    round_trip_MBps=_mbps(nb, sc["device_ms"] + sd["device_ms"]), roundtrip_ok=ok), digests

    for _ in range(max(warmup, 0)):
        dev_round(bufs[:64], cc.FORM_PERSISTENT)
    pick = W.config2_sample(sample)
    sub = [bufs[i] for i in pick]
    plain, dig_p = dev_round(sub, cc.FORM_PLAIN)
    batched_sub, dig_b = dev_round(sub, cc.FORM_PERSISTENT)
    full, dig_full = dev_round(bufs, cc.FORM_PERSISTENT)
    ref = reference_sha256("many4096")
    sha_ok = (dig_full == ref) if ref else None
    ctx.close()
    return {
        "workload": "4096 buffers, log-uniform 4 KiB..4 MiB (%.2f GiB), 0.5 text / 0.25 walk / 0.15 random / "
                    "0.1 runs, 256 KiB chunks, unit 128, device buffers" % (full["bytes"] / 2**30),
        "batched": full,
        "plain_sample": {"sample": "%d buffers, every %d-th in size order (smallest and largest included)"
                                   % (len(pick), len(bufs) // sample),
                         "plain": plain, "batched": batched_sub,
                         "speedup_compress": batched_sub["compress_MBps"] / plain["compress_MBps"],
                         "speedup_decompress": batched_sub["decompress_MBps"] / plain["decompress_MBps"],
                         "speedup_round_trip": batched_sub["round_trip_MBps"] / plain["round_trip_MBps"],
                         "byte_identical": dig_p == dig_b},
        "sha256_match": sha_ok,
        "byte_exact": bool(full["roundtrip_ok"] and plain["roundtrip_ok"] and batched_sub["roundtrip_ok"]
                           and dig_p == dig_b and sha_ok is not False),
    }


def fixed_measure(prelearn=1 << 20, steps=2, total=256 << 20):
    """The fixed-model variant (the paper's section 4.5) on homogeneous data,
    as the paper uses it: `total` bytes of the Markov text (the text of the
    benchmark buffers); a prelearn prefix of `prelearn` bytes trains the model
    on the host, then the remaining bytes (1 MiB chunks, one sequential coder
    each) are coded with it unchanged.  Device time of the chunk coding (the
    host prelearn pass is not in it); the round trip is checked byte for
    byte."""
    import torch
    import cucm_b200 as cc
    from cucm_b200 import workloads as W
    data = W.long_text(total, 7)
    n = data.size
    p = dict(PARAMS, prelearn=prelearn)
    ctx = cc.Context(0)
    d_in = torch.from_numpy(data).cuda()
    cap = cc.lib().cucm_compress_bound(n, cc.default_params(**p))
    d_c = torch.empty(cap, dtype=torch.uint8, device="cuda")
    d_o = torch.empty(n, dtype=torch.uint8, device="cuda")
    tc = td = 0.0
    for i in range(steps + 1):
        m = ctx.compress_dev(d_in.data_ptr(), n, d_c.data_ptr(), cap, fixed=True, **p)
        c_ms = ctx.last_stats()["kernel_ms"]
        ctx.decompress_dev(d_c.data_ptr(), m, d_o.data_ptr(), n)
        d_ms = ctx.last_stats()["kernel_ms"]
        if i:
            tc += c_ms
            td += d_ms
    ok = bool(torch.equal(d_o, d_in))
    ctx.close()
    body = n - prelearn
    return {"workload": "%d MiB of Markov text, %d-byte prelearn prefix, then 1 MiB chunks coded with the fixed "
                        "model" % (total >> 20, prelearn),
            "compress_MBps": _mbps(body * steps, tc), "decompress_MBps": _mbps(body * steps, td),
            "ratio": n / m, "compressed_bytes": int(m), "byte_exact": ok,
            "kernel_ms": {"compress": tc / steps, "decompress": td / steps}}


def run_batch(args):
    """Configs 2 / 3 as a line of their own."""
    r = batch_measure(args.warmup, args.plain_sample)
    line = {"metric": "batched compress+decompress round-trip MB/s", "value": r["batched"]["round_trip_MBps"],
            "unit": "MB/s", "n_gpus": 1, "higher_is_better": True, "dtype": "u8", "data": "synthetic",
            "config": {"workload": r["workload"], "form": "persistent (one launch for all buffers)"}}
    line.update(r)
    print(json.dumps(line), flush=True)


def _pctl(xs, q):
    import numpy as np
    return float(np.percentile(np.asarray(xs), q)) if xs else None


def serve_measure(loads, requests):
    """Config 4: the serving loop under Poisson request streams at the given
    offered loads (GB/s), against serving the same stream one request at a
    time through the single-call API.  The per-request form runs first on a
    context of its own, which is then released, so that the server alone
    holds its HBM budget (120 GB)."""
    import numpy as np
    import torch
    import cucm_b200 as cc
    from cucm_b200 import workloads as W
    ctx = cc.Context(0)
    streams = []
    for li, gbps in enumerate(loads):
        arrivals, comp, bufs, p = W.config4(requests, gbps, seed=4 + li)
        dec_idx = [i for i in range(len(bufs)) if not comp[i]]
        blobs = ctx.compress_many([bufs[i] for i in dec_idx], **p) if dec_idx else []
        inputs = []
        for i, b in enumerate(bufs):
            src = b if comp[i] else np.frombuffer(blobs[dec_idx.index(i)], dtype=np.uint8)
            inputs.append(torch.from_numpy(src.copy()).pin_memory().numpy() if len(src) else src)
        # one request at a time, in arrival order (the plain per-request form)
        lat_p, res_p = [], []
        t0 = time.perf_counter()
        for i in range(len(bufs)):
            d = t0 + arrivals[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            out = ctx.compress(inputs[i], **p) if comp[i] else ctx.decompress(inputs[i])
            lat_p.append((time.perf_counter() - t0 - arrivals[i]) * 1e3)
            res_p.append(out)
        t_plain = time.perf_counter() - t0
        streams.append((gbps, arrivals, comp, bufs, p, inputs, lat_p, res_p, t_plain))
    ctx.close()

    srv = cc.Server(0, hbm_budget=120 * 10**9)
    results = []
    for gbps, arrivals, comp, bufs, p, inputs, lat_p, res_p, t_plain in streams:
        cs = p["chunksize"]
        caps = [cc.many_cap(len(b), cs) if comp[i] else max(len(b), 1) for i, b in enumerate(bufs)]
        outs = [torch.empty(c, dtype=torch.uint8).pin_memory().numpy() for c in caps]
        nbytes = sum(len(b) for b in bufs)
        lat, res = [None] * len(bufs), [None] * len(bufs)
        t0 = time.perf_counter()
        ids = []
        for i in range(len(bufs)):
            d = t0 + arrivals[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            if comp[i]:
                ids.append(srv.submit_compress(inputs[i], out=outs[i], **p))
            else:
                ids.append(srv.submit_decompress(inputs[i], out=outs[i]))
        for i, rid in enumerate(ids):
            st, data, ms = srv.poll(rid, -1)
            if st:
                raise SystemExit("serve request %d failed: %d" % (i, st))
            lat[i], res[i] = ms, data
        t_srv = time.perf_counter() - t0
        exact = all(a == b for a, b in zip(res, res_p)) and all(
            res[i] == bufs[i].tobytes() for i in range(len(bufs)) if not comp[i])
        results.append({"offered_GBps": gbps, "requests": len(bufs), "bytes": nbytes,
                        "serve": {"p50_ms": _pctl(lat, 50), "p99_ms": _pctl(lat, 99),
                                  "sustained_MBps": nbytes / t_srv / 1e6},
                        "one_at_a_time": {"p50_ms": _pctl(lat_p, 50), "p99_ms": _pctl(lat_p, 99),
                                          "sustained_MBps": nbytes / t_plain / 1e6},
                        "byte_exact": bool(exact)})
    info = srv.stats()
    srv.close()
    return {"workload": "Poisson request streams, %d requests per load, sizes log-uniform 1 KiB..16 MiB, "
                        "70%% compress / 30%% decompress, content as the 4096-buffer set, 256 KiB chunks, "
                        "HBM budget 120 GB; latency from submit to result on the host" % requests,
            "slots": info["slots"], "levels": results,
            "byte_exact": all(r["byte_exact"] for r in results)}


def run_fixed(args):
    """The fixed-model variant as a line of its own."""
    r = fixed_measure()
    line = {"metric": "fixed-model compress+decompress MB/s", "unit": "MB/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "u8", "data": "synthetic", "config": {"workload": r["workload"]}}
    line.update(r)
    print(json.dumps(line), flush=True)


def run_serve(args):
    """Config 4 as a line of its own."""
    r = serve_measure([float(x) for x in args.loads.split(",")], args.requests)
    best = max(x["serve"]["sustained_MBps"] for x in r["levels"])
    line = {"metric": "serving sustained MB/s and p50/p99 latency", "value": best, "unit": "MB/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "u8", "data": "synthetic",
            "config": {"workload": r["workload"], "slots": r["slots"]}}
    line.update(r)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
