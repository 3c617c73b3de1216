"""ctypes binding of the CPU restatement (oracle/cucm_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker.  The product never imports it.
"""
import ctypes
import functools
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libcucm_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")


def build():
    subprocess.run(["make", "-s", "-C", HERE, "libcucm_oracle.so", "oracle_cli"], check=True)


@functools.lru_cache(maxsize=1)
def lib():
    if not os.path.exists(LIB):
        build()
    L = ctypes.CDLL(LIB)
    u8pp = ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8))
    L.co_compress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t,
                              ctypes.c_int, ctypes.c_int, u8pp, ctypes.POINTER(ctypes.c_size_t)]
    L.co_compress.restype = ctypes.c_int
    L.co_compress_ex.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int, u8pp, ctypes.POINTER(ctypes.c_size_t)]
    L.co_compress_ex.restype = ctypes.c_int
    L.co_decompress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, u8pp, ctypes.POINTER(ctypes.c_size_t)]
    L.co_decompress.restype = ctypes.c_int
    L.co_tables.argtypes = [ctypes.c_void_p] * 3
    L.co_next_state_table.restype = ctypes.POINTER(ctypes.c_uint8)
    libc = ctypes.CDLL(None)
    libc.free.argtypes = [ctypes.c_void_p]
    L._free = libc.free
    return L


def _ptr(data):
    b = bytes(data)
    buf = ctypes.create_string_buffer(b, max(len(b), 1))
    return buf, len(b)


def _take(p, n):
    out = ctypes.string_at(p, n.value) if n.value else b""
    lib()._free(ctypes.cast(p, ctypes.c_void_p))
    return out


def compress(data, chunksize=1 << 20, unit=128, prelearn=0, batch=100, threads=0, fixed=False):
    """Whole container, the reference's output for `cucm_compress -s -u -p -b`
    (with `fixed`, the fixed-model variant of the paper's section 4.5)."""
    buf, n = _ptr(data)
    out = ctypes.POINTER(ctypes.c_uint8)()
    on = ctypes.c_size_t()
    rc = lib().co_compress_ex(buf, n, chunksize, unit, prelearn, batch, 1 if fixed else 0, threads,
                              ctypes.byref(out), ctypes.byref(on))
    if rc:
        raise RuntimeError("oracle compress failed: %d" % rc)
    return _take(out, on)


def decompress(blob, threads=0):
    buf, n = _ptr(blob)
    out = ctypes.POINTER(ctypes.c_uint8)()
    on = ctypes.c_size_t()
    rc = lib().co_decompress(buf, n, threads, ctypes.byref(out), ctypes.byref(on))
    if rc:
        raise RuntimeError("oracle decompress failed: %d" % rc)
    return _take(out, on)


def tables():
    import numpy as np
    sq = np.zeros(4096, np.int32)
    st = np.zeros(4096, np.int32)
    dt = np.zeros(1024, np.int32)
    lib().co_tables(sq.ctypes.data, st.ctypes.data, dt.ctypes.data)
    nex = np.ctypeslib.as_array(lib().co_next_state_table(), shape=(512,)).reshape(256, 2).copy()
    return sq, st, dt, nex


def ref_binary(name):
    """Path of a reference binary built by make_ref.py, or None."""
    p = os.path.join(REF_DIR, name)
    return p if os.path.exists(p) else None
