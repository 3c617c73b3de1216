"""In-tree build of the CUDA library and the command-line tools.

Produces, next to this file:
  libcucm.so             the C-ABI library (include/cucm.h), sm_100a only
  bin/cucm_compress      drop-in for the reference's compressor CLI
  bin/cucm_decompress    drop-in for the reference's decompressor CLI
  libcucm_workload.so    synthetic workload generator used by bench/tests

Run:  python -m cucm_b200.build [--force]
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
BIN = os.path.join(PKG, "bin")
LIB = os.path.join(PKG, "libcucm.so")
WORKLOAD_LIB = os.path.join(PKG, "libcucm_workload.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
           "-I" + os.path.join(ROOT, "include")]
CU_SOURCES = ["engine_kernels.cu", "api.cu", "serve.cu", "noalloc.cu", "autotune.cu"]
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".cuh", ".h")))


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "cucm.h"), __file__]
    objs, jobs = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            jobs.append([nvcc()] + ARCH + NVFLAGS + ["-c", s, "-o", o])
    if jobs:
        with cf.ThreadPoolExecutor(len(jobs)) as ex:
            for r in ex.map(_run, jobs):
                if verbose:
                    sys.stdout.write(r.stderr)
    if force or _stale(LIB, objs):
        _run([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    for name in ("cli_compress", "cli_decompress"):
        exe = os.path.join(BIN, name.replace("cli_", "cucm_"))
        src = os.path.join(CSRC, name + ".cpp")
        if force or _stale(exe, [src, LIB] + hdrs):
            _run([nvcc(), "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-o", exe, src,
                  "-L" + PKG, "-lcucm", "-Xlinker", "-rpath=$ORIGIN/.."])
    wsrc = os.path.join(CSRC, "workload_gen.c")
    if os.path.exists(wsrc) and (force or _stale(WORKLOAD_LIB, [wsrc])):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-o", WORKLOAD_LIB, wsrc])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
