"""cucm_b200 -- Python face of the B200 CuCM coder (libcucm.so, include/cucm.h).

The reference (OceanCT/CuCM) exposes its hot path as host functions inside
two CUDA programs; this module binds the C ABI that replaces them and keeps
their names and argument meaning:

  compress_batch(data, chunksize, unitlength)        compress_batch,  cucm_compress_v2.cu:990
  decompressbatch(body, out_size, chunksize, unit)   decompressbatch, cucm_decompress_v2.cu:898
  compress_file(in_path, out_path, ...)              compress_file,   cucm_compress_v2.cu:1151
  decompress(in_path, out_path)                      decompress,      cucm_decompress_v2.cu:1185

plus whole-buffer compress()/decompress() and a Context for repeated calls.
Everything runs on the GPU through libcucm.so; there is no CPU fallback, and
a missing or unloadable library raises instead of degrading.
"""
import ctypes
import functools
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
# the in-tree build; CUCM_LIBRARY names another build of the same library
LIB_PATH = os.environ.get("CUCM_LIBRARY") or os.path.join(_PKG, "libcucm.so")

FORM_AUTO, FORM_PLAIN, FORM_PERSISTENT = 0, 1, 2

CUCM_OK = 0
EINVAL, ENOSPC, EFORMAT, EMISMATCH = -1, -2, -3, -10
PENDING = 1
OP_COMPRESS, OP_DECOMPRESS = 0, 1
_ERRORS = {
    -1: "EINVAL", -2: "ENOSPC", -3: "EFORMAT", -4: "ENOMEM", -5: "ECUDA",
    -6: "ENODEV", -7: "ETIMEOUT", -8: "EBUSY", -9: "ENOTFOUND", -10: "EMISMATCH",
}


class CucmError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = lib().cucm_strerror(status).decode()
        super().__init__("%s: %s (%s)" % (what or "cucm", msg, _ERRORS.get(status, status)))


FORMAT_AUTO, FORMAT_32, FORMAT_64 = 0, 1, 2


class Params(ctypes.Structure):
    _fields_ = [("chunksize", ctypes.c_uint64), ("unit", ctypes.c_uint32),
                ("prelearn", ctypes.c_uint64), ("batch", ctypes.c_uint32), ("format", ctypes.c_uint32),
                ("fixed_model", ctypes.c_uint32)]


class Stats(ctypes.Structure):
    _fields_ = [("device_ms", ctypes.c_double), ("kernel_ms", ctypes.c_double),
                ("launches", ctypes.c_uint64), ("chunks", ctypes.c_uint64)]


class ServerInfo(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_uint64), ("budget", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("bytes_in", ctypes.c_uint64), ("bytes_out", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("queued", ctypes.c_uint64), ("inflight", ctypes.c_uint64)]


class Tuning(ctypes.Structure):
    _fields_ = [("form", ctypes.c_int), ("spec_bits", ctypes.c_int),
                ("max_slots", ctypes.c_int), ("hbm_budget", ctypes.c_uint64), ("kernel", ctypes.c_int),
                ("dec_pairs", ctypes.c_int), ("dec_tables", ctypes.c_int), ("cmp_ctas", ctypes.c_int),
                ("dec_spin_limit", ctypes.c_uint32)]


def make_tuning(form=FORM_AUTO, spec_bits=0, max_slots=0, hbm_budget=0, kernel=0, dec_pairs=0, dec_tables=0,
                cmp_ctas=0, dec_spin_limit=0):
    """A cucm_tuning; 0 everywhere means the derived defaults."""
    return Tuning(form, spec_bits, max_slots, hbm_budget, kernel, dec_pairs, dec_tables, cmp_ctas, dec_spin_limit)


class TuneResult(ctypes.Structure):
    _fields_ = [("tuning", Tuning), ("compress_ms", ctypes.c_double), ("decompress_ms", ctypes.c_double)]


def _tuning_dict(t):
    return {f: getattr(t, f) for f, _ in Tuning._fields_}


_u8p = ctypes.POINTER(ctypes.c_uint8)
_u64p = ctypes.POINTER(ctypes.c_uint64)

# (name, restype, argtypes) for every entry point of include/cucm.h
SIGNATURES = [
    ("cucm_default_params", None, [ctypes.POINTER(Params)]),
    ("cucm_strerror", ctypes.c_char_p, [ctypes.c_int]),
    ("cucm_version", ctypes.c_char_p, []),
    ("cucm_ctx_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Tuning), ctypes.POINTER(ctypes.c_void_p)]),
    ("cucm_ctx_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("cucm_ctx_set_tuning", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Tuning)]),
    ("cucm_ctx_get_tuning", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Tuning)]),
    ("cucm_autotune", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Params),
                                     ctypes.c_int, ctypes.POINTER(TuneResult), ctypes.c_uint32,
                                     ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(Tuning)]),
    ("cucm_compress_bound", ctypes.c_uint64, [ctypes.c_uint64, ctypes.POINTER(Params)]),
    ("cucm_decompressed_size", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, _u64p]),
    ("cucm_compress", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Params),
                                     ctypes.c_void_p, ctypes.c_uint64, _u64p]),
    ("cucm_decompress", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                       ctypes.c_uint64, _u64p]),
    ("cucm_compress_dev", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Params),
                                         ctypes.c_void_p, ctypes.c_uint64, _u64p]),
    ("cucm_decompress_dev", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                           ctypes.c_uint64, _u64p]),
    ("cucm_compress_batch", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                           ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, _u64p]),
    ("cucm_decompress_batch", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                             ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64]),
    ("cucm_model_prelearn", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    ("cucm_model_from_container", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    ("cucm_model_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("cucm_compress_batch_model", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                                 ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                                 _u64p]),
    ("cucm_decompress_batch_model", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                                   ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_uint64]),
    ("cucm_compress_batch_dev", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                               ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                               _u64p]),
    ("cucm_frame_bodies", ctypes.c_int, [ctypes.POINTER(Params), ctypes.c_uint64, ctypes.c_uint32,
                                         ctypes.POINTER(ctypes.c_void_p), _u64p, ctypes.POINTER(ctypes.c_uint32),
                                         ctypes.c_void_p, ctypes.c_uint64, _u64p]),
    ("cucm_frame_bodies_dev", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Params), ctypes.c_uint64,
                                             ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p), _u64p,
                                             ctypes.POINTER(ctypes.c_uint32), ctypes.c_void_p, ctypes.c_uint64,
                                             _u64p]),
    ("cucm_decompress_range_dev", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                                 ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                                                 ctypes.c_uint64, _u64p]),
    ("cucm_compress_many", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p), _u64p,
                                          ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_void_p), _u64p, _u64p,
                                          ctypes.POINTER(ctypes.c_int)]),
    ("cucm_decompress_many", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p), _u64p,
                                            ctypes.POINTER(ctypes.c_void_p), _u64p, _u64p,
                                            ctypes.POINTER(ctypes.c_int)]),
    ("cucm_compress_many_dev", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p),
                                              _u64p, ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_void_p), _u64p,
                                              _u64p, ctypes.POINTER(ctypes.c_int)]),
    ("cucm_decompress_many_dev", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p),
                                                _u64p, ctypes.POINTER(ctypes.c_void_p), _u64p, _u64p,
                                                ctypes.POINTER(ctypes.c_int)]),
    ("cucm_server_create", ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(Tuning),
                                          ctypes.POINTER(ctypes.c_void_p)]),
    ("cucm_server_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("cucm_serve_submit", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                         ctypes.POINTER(Params), ctypes.c_void_p, ctypes.c_uint64, _u64p]),
    ("cucm_serve_poll", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                       _u64p, ctypes.POINTER(ctypes.c_double)]),
    ("cucm_server_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerInfo)]),
    ("cucm_server_set_queue_limit", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    ("cucm_last_device_ms", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    ("cucm_last_launches", ctypes.c_int, [ctypes.c_void_p, _u64p]),
    ("cucm_last_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Stats)]),
    ("cucm_compress_chunk_noalloc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                                   ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, _u64p,
                                                   ctypes.c_void_p]),
]


@functools.lru_cache(maxsize=1)
def lib():
    """Load libcucm.so (built in-tree by cucm_b200.build)."""
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libcucm.so is not built; run `python -m cucm_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


def default_params(chunksize=None, unit=None, prelearn=None, batch=None, fmt=None, fixed=None):
    """cucm_params: the reference CLI's defaults, then the given fields; fmt
    is the container format (FORMAT_AUTO, FORMAT_32 or FORMAT_64), fixed the
    fixed-model variant (needs a prelearn prefix)."""
    p = Params()
    lib().cucm_default_params(ctypes.byref(p))
    if fixed is not None:
        p.fixed_model = 1 if fixed else 0
    if fmt is not None:
        p.format = int(fmt)
    if chunksize is not None:
        p.chunksize = int(chunksize)
    if unit is not None:
        p.unit = int(unit)
    if prelearn is not None:
        p.prelearn = int(prelearn)
    if batch is not None:
        p.batch = int(batch)
    return p


def many_cap(n, chunksize, prelearn=0):
    """An output capacity that nearly every container of n input bytes fits:
    up to 2x plus 4 KiB per chunk.  A chunk shorter than the chunk size still
    codes the stale model buffer up to the chunk end, as the reference does,
    so even a tiny input can need about a chunk's worth.  The batched calls
    redo the rare container that needs more."""
    nchunks = (max(n - prelearn, 0) + chunksize - 1) // chunksize
    return 64 + prelearn * 8 + nchunks * (8 + 2 * chunksize + 4096)


def _buf_w(arr):
    """(pointer, capacity, keepalive) of a writable numpy uint8 array."""
    import numpy as np
    a = arr.view(np.uint8).reshape(-1)
    return a.ctypes.data, a.size, a


def _buf(data):
    """(pointer, length, keepalive) for bytes-like or numpy input."""
    try:
        import numpy as np
        if isinstance(data, np.ndarray):
            a = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
            return a.ctypes.data, a.size, a
    except ImportError:  # pragma: no cover
        pass
    b = bytes(data)
    cb = ctypes.create_string_buffer(b, len(b)) if b else ctypes.create_string_buffer(1)
    return ctypes.addressof(cb), len(b), cb


class Model:
    """An initial model (the reference's sm_init / mixer_init): trained by
    the prelearn pass over a prefix, or read from a container's prelearn
    block.  Host memory only; pass it to compress_batch / decompressbatch."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def prelearn(cls, prefix):
        ptr, n, keep = _buf(prefix)
        h = ctypes.c_void_p()
        rc = lib().cucm_model_prelearn(ptr, n, ctypes.byref(h))
        if rc:
            raise CucmError(rc, "cucm_model_prelearn")
        return cls(h)

    @classmethod
    def from_container(cls, blob):
        """The container's model, or None when it has no prelearn block."""
        ptr, n, keep = _buf(blob)
        h = ctypes.c_void_p()
        rc = lib().cucm_model_from_container(ptr, n, ctypes.byref(h))
        if rc:
            raise CucmError(rc, "cucm_model_from_container")
        return cls(h) if h.value else None

    def close(self):
        if self._h:
            lib().cucm_model_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One CUDA device, one stream and the device pools of the coder."""

    def __init__(self, device=0, **tuning):
        self._h = ctypes.c_void_p()
        t = make_tuning(**tuning)
        rc = lib().cucm_ctx_create(int(device), ctypes.byref(t), ctypes.byref(self._h))
        if rc:
            raise CucmError(rc, "cucm_ctx_create")

    def close(self):
        if self._h:
            lib().cucm_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tuning(self, **tuning):
        """Replace the execution choices (make_tuning's keywords; omitted = 0)."""
        t = make_tuning(**tuning)
        rc = lib().cucm_ctx_set_tuning(self._h, ctypes.byref(t))
        if rc:
            raise CucmError(rc, "cucm_ctx_set_tuning")

    def get_tuning(self):
        t = Tuning()
        rc = lib().cucm_ctx_get_tuning(self._h, ctypes.byref(t))
        if rc:
            raise CucmError(rc, "cucm_ctx_get_tuning")
        return _tuning_dict(t)

    def autotune(self, sample, reps=1, chunksize=1 << 20, unit=128, prelearn=0, batch=100):
        """Measure every execution choice on `sample` (cucm_autotune), apply
        the fastest and return (chosen tuning, [measured candidates])."""
        p = default_params(chunksize, unit, prelearn, batch)
        ptr, n, keep = _buf(sample)
        res = (TuneResult * 64)()
        count = ctypes.c_uint32()
        best = Tuning()
        rc = lib().cucm_autotune(self._h, ptr, n, ctypes.byref(p), int(reps), res, 64, ctypes.byref(count),
                                 ctypes.byref(best))
        if rc:
            raise CucmError(rc, "cucm_autotune")
        cands = [dict(_tuning_dict(r.tuning), compress_ms=r.compress_ms, decompress_ms=r.decompress_ms)
                 for r in res[:min(count.value, 64)]]
        return _tuning_dict(best), cands

    def compress(self, data, chunksize=1 << 20, unit=128, prelearn=0, batch=100, fmt=FORMAT_AUTO, out=None,
                 fixed=False):
        """The container of `data`.  With `out` (a writable numpy uint8 array)
        the container is written there and a view of it returned; otherwise
        bytes, in a buffer of the compress bound.  `fixed`: the fixed-model
        variant (prelearn > 0)."""
        p = default_params(chunksize, unit, prelearn, batch, fmt, fixed)
        ptr, n, keep = _buf(data)
        got = ctypes.c_uint64()
        if out is not None:
            optr, cap, out = _buf_w(out)
            rc = lib().cucm_compress(self._h, ptr, n, ctypes.byref(p), optr, cap, ctypes.byref(got))
            if rc:
                raise CucmError(rc, "cucm_compress")
            return out[:got.value]
        cap = lib().cucm_compress_bound(n, ctypes.byref(p))
        buf = ctypes.create_string_buffer(max(cap, 1))
        rc = lib().cucm_compress(self._h, ptr, n, ctypes.byref(p), buf, cap, ctypes.byref(got))
        if rc:
            raise CucmError(rc, "cucm_compress")
        return buf.raw[:got.value]

    def decompress(self, blob, out=None):
        """The original bytes of a container; into `out` (a writable numpy
        uint8 array, returned as a view) when given."""
        ptr, n, keep = _buf(blob)
        size = ctypes.c_uint64()
        rc = lib().cucm_decompressed_size(ptr, n, ctypes.byref(size))
        if rc:
            raise CucmError(rc, "cucm_decompressed_size")
        got = ctypes.c_uint64()
        if out is not None:
            optr, cap, out = _buf_w(out)
            rc = lib().cucm_decompress(self._h, ptr, n, optr, cap, ctypes.byref(got))
            if rc:
                raise CucmError(rc, "cucm_decompress")
            return out[:got.value]
        buf = ctypes.create_string_buffer(max(size.value, 1))
        rc = lib().cucm_decompress(self._h, ptr, n, buf, size.value, ctypes.byref(got))
        if rc:
            raise CucmError(rc, "cucm_decompress")
        return buf.raw[:got.value]

    def compress_dev(self, d_in, n, d_out, cap, chunksize=1 << 20, unit=128, prelearn=0, batch=100,
                     fmt=FORMAT_AUTO, fixed=False):
        """Device pointers in and out; returns the container size."""
        p = default_params(chunksize, unit, prelearn, batch, fmt, fixed)
        got = ctypes.c_uint64()
        rc = lib().cucm_compress_dev(self._h, d_in, n, ctypes.byref(p), d_out, cap, ctypes.byref(got))
        if rc:
            raise CucmError(rc, "cucm_compress_dev")
        return got.value

    def decompress_dev(self, d_in, n, d_out, cap):
        got = ctypes.c_uint64()
        rc = lib().cucm_decompress_dev(self._h, d_in, n, d_out, cap, ctypes.byref(got))
        if rc:
            raise CucmError(rc, "cucm_decompress_dev")
        return got.value

    def compress_batch(self, data, chunksize, unitlength=128, model=None):
        """Batch body of `data` (compress_batch); `model` is sm_init/mixer_init
        (a Model, or None for the zero model)."""
        ptr, n, keep = _buf(data)
        nchunks = (n + chunksize - 1) // chunksize
        cap = nchunks * (4 + 32 * chunksize + 1) + 16
        out = ctypes.create_string_buffer(max(cap, 1))
        got = ctypes.c_uint64()
        rc = lib().cucm_compress_batch_model(self._h, ptr, n, chunksize, unitlength, model._h if model else None,
                                             out, cap, ctypes.byref(got))
        if rc:
            raise CucmError(rc, "cucm_compress_batch_model")
        return out.raw[:got.value]

    def decompressbatch(self, body, out_size, chunksize, unitlength=128, model=None):
        ptr, n, keep = _buf(body)
        out = ctypes.create_string_buffer(max(out_size, 1))
        rc = lib().cucm_decompress_batch_model(self._h, ptr, n, chunksize, unitlength, model._h if model else None,
                                               out, out_size)
        if rc:
            raise CucmError(rc, "cucm_decompress_batch_model")
        return out.raw[:out_size]

    def compress_many(self, buffers, chunksize=1 << 20, unit=128, prelearn=0, batch=100):
        """Containers of many buffers in one call (the batched form); each is
        byte-identical to compress() of that buffer alone."""
        p = default_params(chunksize, unit, prelearn, batch)
        k = len(buffers)
        bufs = [_buf(b) for b in buffers]
        ins = (ctypes.c_void_p * k)(*[b[0] for b in bufs])
        ns = (ctypes.c_uint64 * k)(*[b[1] for b in bufs])
        # optimistic output sizes; entries that need more are redone alone
        caps = [min(lib().cucm_compress_bound(b[1], ctypes.byref(p)), many_cap(b[1], chunksize)) for b in bufs]
        outs_b = [ctypes.create_string_buffer(max(c, 1)) for c in caps]
        outs = (ctypes.c_void_p * k)(*[ctypes.addressof(o) for o in outs_b])
        capa = (ctypes.c_uint64 * k)(*caps)
        got = (ctypes.c_uint64 * k)()
        st = (ctypes.c_int * k)()
        rc = lib().cucm_compress_many(self._h, k, ins, ns, ctypes.byref(p), outs, capa, got, st)
        res = []
        for i in range(k):
            if st[i] == ENOSPC:
                res.append(self.compress(buffers[i], chunksize, unit, prelearn, batch))
            elif st[i]:
                raise CucmError(st[i], "cucm_compress_many")
            else:
                res.append(outs_b[i].raw[:got[i]])
        if rc and rc != ENOSPC:
            raise CucmError(rc, "cucm_compress_many")
        return res

    def decompress_many(self, blobs):
        k = len(blobs)
        bufs = [_buf(b) for b in blobs]
        sizes = []
        for p_, n_, _ in bufs:
            s = ctypes.c_uint64()
            rc = lib().cucm_decompressed_size(p_, n_, ctypes.byref(s))
            if rc:
                raise CucmError(rc, "cucm_decompressed_size")
            sizes.append(s.value)
        ins = (ctypes.c_void_p * k)(*[b[0] for b in bufs])
        ns = (ctypes.c_uint64 * k)(*[b[1] for b in bufs])
        outs_b = [ctypes.create_string_buffer(max(s, 1)) for s in sizes]
        outs = (ctypes.c_void_p * k)(*[ctypes.addressof(o) for o in outs_b])
        capa = (ctypes.c_uint64 * k)(*sizes)
        got = (ctypes.c_uint64 * k)()
        st = (ctypes.c_int * k)()
        rc = lib().cucm_decompress_many(self._h, k, ins, ns, outs, capa, got, st)
        if rc:
            raise CucmError(rc, "cucm_decompress_many")
        return [outs_b[i].raw[:got[i]] for i in range(k)]

    def compress_many_dev(self, ins, outs, chunksize=1 << 20, unit=128, prelearn=0, batch=100):
        """Batched form on device buffers.  ins: [(device ptr, bytes)],
        outs: [(device ptr, capacity)].  Returns (sizes, statuses)."""
        p = default_params(chunksize, unit, prelearn, batch)
        return self._many_dev(lib().cucm_compress_many_dev, ins, outs, ctypes.byref(p))

    def decompress_many_dev(self, ins, outs):
        """Batched decompression on device buffers; see compress_many_dev."""
        return self._many_dev(lib().cucm_decompress_many_dev, ins, outs, None)

    def _many_dev(self, fn, ins, outs, params):
        k = len(ins)
        a_in = (ctypes.c_void_p * k)(*[int(x[0]) for x in ins])
        a_n = (ctypes.c_uint64 * k)(*[int(x[1]) for x in ins])
        a_out = (ctypes.c_void_p * k)(*[int(x[0]) for x in outs])
        a_cap = (ctypes.c_uint64 * k)(*[int(x[1]) for x in outs])
        got = (ctypes.c_uint64 * k)()
        st = (ctypes.c_int * k)()
        if params is None:
            rc = fn(self._h, k, a_in, a_n, a_out, a_cap, got, st)
        else:
            rc = fn(self._h, k, a_in, a_n, params, a_out, a_cap, got, st)
        if rc and rc != ENOSPC:
            raise CucmError(rc, fn.__name__)
        return list(got), list(st)

    def last_device_ms(self):
        v = ctypes.c_double()
        lib().cucm_last_device_ms(self._h, ctypes.byref(v))
        return v.value

    def last_launches(self):
        v = ctypes.c_uint64()
        lib().cucm_last_launches(self._h, ctypes.byref(v))
        return v.value

    def last_stats(self):
        st = Stats()
        lib().cucm_last_stats(self._h, ctypes.byref(st))
        return dict(device_ms=st.device_ms, kernel_ms=st.kernel_ms, launches=st.launches, chunks=st.chunks)


def frame_bodies(bodies, counts, orig_size, chunksize=1 << 20, unit=128, batch=100, fmt=FORMAT_AUTO):
    """The container of a stream whose chunks were coded in consecutive
    pieces (cucm_frame_bodies; host buffers, no device work): bodies[i] is the
    batch body of counts[i] consecutive chunks."""
    p = default_params(chunksize, unit, 0, batch, fmt)
    k = len(bodies)
    bufs = [_buf(b) for b in bodies]
    ptrs = (ctypes.c_void_p * k)(*[b[0] for b in bufs])
    ns = (ctypes.c_uint64 * k)(*[b[1] for b in bufs])
    cs = (ctypes.c_uint32 * k)(*counts)
    cap = 64 + 8 * ((sum(counts) + batch - 1) // batch) + 4 * sum(counts) + sum(b[1] for b in bufs)
    out = ctypes.create_string_buffer(cap)
    got = ctypes.c_uint64()
    rc = lib().cucm_frame_bodies(ctypes.byref(p), orig_size, k, ptrs, ns, cs, out, cap, ctypes.byref(got))
    if rc:
        raise CucmError(rc, "cucm_frame_bodies")
    return out.raw[:got.value]


_default_ctx = None


def _ctx():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def compress(data, chunksize=1 << 20, unit=128, prelearn=0, batch=100):
    """Whole container, byte-identical to the reference CLI's output."""
    return _ctx().compress(data, chunksize, unit, prelearn, batch)


def decompress(blob):
    return _ctx().decompress(blob)


def compress_batch(data, chunksize, unitlength=128):
    """Batch body (big-endian chunk end offsets + payloads) of `data`, coded
    from the zero model, as compress_batch() returns it."""
    return _ctx().compress_batch(data, chunksize, unitlength)


def decompressbatch(body, out_size, chunksize, unitlength=128):
    return _ctx().decompressbatch(body, out_size, chunksize, unitlength)


def compress_file(in_path, out_path, chunksize=1 << 20, unitlength=128, prelearn_size=0, batch_num=100,
                  chunknum=-1):
    with open(in_path, "rb") as f:
        data = f.read()
    if chunknum > 0:
        data = data[:chunksize * chunknum]
    blob = compress(data, chunksize, unitlength, prelearn_size, batch_num)
    with open(out_path, "wb") as f:
        f.write(blob)
    return len(blob)


def decompress_file(in_path, out_path):
    with open(in_path, "rb") as f:
        blob = f.read()
    data = decompress(blob)
    with open(out_path, "wb") as f:
        f.write(data)
    return len(data)


class Server:
    """The serving loop (cucm_server_*): submit compress / decompress requests
    from any thread, poll for their results.  Requests that arrive while
    others run are admitted as chunk slots and memory free up, and share
    launches that overlap on the device; every result equals the
    single-call API's."""

    def __init__(self, device=0, hbm_budget=0, max_slots=0, kernel=0):
        self._h = ctypes.c_void_p()
        t = make_tuning(form=FORM_PERSISTENT, max_slots=max_slots, hbm_budget=hbm_budget, kernel=kernel)
        rc = lib().cucm_server_create(device, hbm_budget, ctypes.byref(t), ctypes.byref(self._h))
        if rc:
            raise CucmError(rc, "cucm_server_create")
        self._live = {}

    def submit_compress(self, data, chunksize=1 << 20, unit=128, prelearn=0, batch=100, out=None):
        """Queue a compression; `out` (optional, e.g. pinned) receives the container."""
        p = default_params(chunksize, unit, prelearn, batch)
        ptr, n, keep = _buf(data)
        if out is None:
            out = ctypes.create_string_buffer(max(many_cap(n, chunksize, prelearn), 1))
            optr, cap = ctypes.addressof(out), len(out)
        else:
            optr, cap, out = _buf_w(out)
        rid = ctypes.c_uint64()
        rc = lib().cucm_serve_submit(self._h, OP_COMPRESS, ptr, n, ctypes.byref(p), optr, cap, ctypes.byref(rid))
        if rc:
            raise CucmError(rc, "cucm_serve_submit")
        self._live[rid.value] = (keep, out, optr)
        return rid.value

    def submit_decompress(self, blob, out=None):
        """Queue a decompression; `out` (optional) receives the original bytes."""
        ptr, n, keep = _buf(blob)
        size = ctypes.c_uint64()
        rc = lib().cucm_decompressed_size(ptr, n, ctypes.byref(size))
        if rc:
            raise CucmError(rc, "cucm_decompressed_size")
        if out is None:
            out = ctypes.create_string_buffer(max(size.value, 1))
            optr, cap = ctypes.addressof(out), size.value
        else:
            optr, cap, out = _buf_w(out)
        rid = ctypes.c_uint64()
        rc = lib().cucm_serve_submit(self._h, OP_DECOMPRESS, ptr, n, None, optr, cap, ctypes.byref(rid))
        if rc:
            raise CucmError(rc, "cucm_serve_submit")
        self._live[rid.value] = (keep, out, optr)
        return rid.value

    def poll(self, rid, timeout_ms=-1):
        """None while pending, else (status, output bytes or None, latency ms)."""
        st = ctypes.c_int()
        n = ctypes.c_uint64()
        lat = ctypes.c_double()
        rc = lib().cucm_serve_poll(self._h, rid, int(timeout_ms), ctypes.byref(st), ctypes.byref(n),
                                   ctypes.byref(lat))
        if rc == PENDING:
            return None
        if rc:
            raise CucmError(rc, "cucm_serve_poll")
        keep, out, optr = self._live.pop(rid)
        data = ctypes.string_at(optr, n.value) if st.value == 0 else None
        return st.value, data, lat.value

    def set_queue_limit(self, limit):
        rc = lib().cucm_server_set_queue_limit(self._h, int(limit))
        if rc:
            raise CucmError(rc, "cucm_server_set_queue_limit")

    def stats(self):
        info = ServerInfo()
        rc = lib().cucm_server_stats(self._h, ctypes.byref(info))
        if rc:
            raise CucmError(rc, "cucm_server_stats")
        return {f: getattr(info, f) for f, _ in ServerInfo._fields_}

    def close(self):
        if self._h:
            lib().cucm_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
