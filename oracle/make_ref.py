#!/usr/bin/env python3
"""Build recipe for oracle/_ref: the reference's own code, compiled here.

Test infrastructure only.  Reads the two reference sources where they lie
(``<reference>/cucm_compress_v2.cu`` and ``<reference>/cucm_decompress_v2.cu``)
and produces, inside ``oracle/_ref/`` only (git-ignored):

* ``cucm_compress_ref`` / ``cucm_decompress_ref`` -- host (CPU) builds made
  with g++ through ``oracle/ref_shim.h``.  The only source rewrites are
  mechanical: the cub/thrust includes are dropped (the shim provides the one
  cub call, an inclusive prefix sum) and every ``k<<<g, b>>>(args);`` launch
  becomes ``shim_launch(g, b, [&] { k(args); });``.  Nothing else of the
  reference is touched, so these binaries execute the reference's own
  kernels, host drivers, container writer/reader and CLI.
* ``cucm_compress_gpu`` / ``cucm_decompress_gpu`` (only with ``--gpu``) --
  the unmodified sources built by nvcc for sm_100a, the reference's own CUDA
  build for the B200.

The rewritten translation units are written to ``oracle/_ref/`` as well and
are never committed.

Usage:  python oracle/make_ref.py [--reference DIR] [--gpu] [--force]
"""
import argparse
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# $CUCM_REFERENCE_DIR, else a sibling checkout named "reference" next to the repository.
DEFAULT_REF = os.environ.get("CUCM_REFERENCE_DIR") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
SOURCES = {
    "cucm_compress": "cucm_compress_v2.cu",
    "cucm_decompress": "cucm_decompress_v2.cu",
}

LAUNCH = re.compile(r"(\w+)\s*<<<(.*?)>>>\s*\((.*?)\)\s*;", re.S)


def rewrite(src: str) -> str:
    lines = []
    for line in src.splitlines():
        s = line.strip()
        if s.startswith("#include") and ("cub/" in s or "thrust/" in s):
            continue
        lines.append(line)
    body = "\n".join(lines) + "\n"

    def repl(m):
        kern, cfg, args = m.group(1), m.group(2), m.group(3)
        grid, block = [c.strip() for c in cfg.split(",")[:2]]
        return "shim_launch((%s), (%s), [&] { %s(%s); });" % (grid, block, kern, args)

    body, n = LAUNCH.subn(repl, body)
    if n == 0:
        raise RuntimeError("no kernel launches found; unexpected source")
    head = ('#include "%s"\n' % os.path.join(HERE, "ref_shim.h")
            + "shim_dim3 blockIdx, threadIdx, blockDim, gridDim;\n")
    return head + body


def newer(target, *deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build_host(ref_dir, force=False):
    os.makedirs(OUT, exist_ok=True)
    built = []
    for name, fname in SOURCES.items():
        src_path = os.path.join(ref_dir, fname)
        exe = os.path.join(OUT, name + "_ref")
        shim = os.path.join(HERE, "ref_shim.h")
        if not force and newer(exe, src_path, shim, __file__):
            built.append(exe)
            continue
        with open(src_path, "r", encoding="utf-8", errors="replace") as f:
            text = f.read()
        cpp = os.path.join(OUT, name + "_ref.cpp")
        with open(cpp, "w") as f:
            f.write(rewrite(text))
        cmd = ["g++", "-O2", "-std=c++17", "-w", "-o", exe, cpp]
        subprocess.run(cmd, check=True)
        built.append(exe)
    return built


def build_gpu(ref_dir, force=False):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    os.makedirs(OUT, exist_ok=True)
    built = []
    for name, fname in SOURCES.items():
        src_path = os.path.join(ref_dir, fname)
        exe = os.path.join(OUT, name + "_gpu")
        if not force and newer(exe, src_path, __file__):
            built.append(exe)
            continue
        cmd = [nvcc, "-O3", "-std=c++17", "-w",
               "-gencode", "arch=compute_100a,code=sm_100a",
               "-o", exe, src_path]
        subprocess.run(cmd, check=True)
        built.append(exe)
    return built


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REF)
    ap.add_argument("--gpu", action="store_true", help="also build the unmodified nvcc sm_100a binaries")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    if not os.path.isdir(a.reference):
        print("reference sources not present at %s; nothing to build" % a.reference)
        return 0
    for p in build_host(a.reference, a.force):
        print(p)
    if a.gpu:
        for p in build_gpu(a.reference, a.force):
            print(p)
    return 0


if __name__ == "__main__":
    sys.exit(main())
