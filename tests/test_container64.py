"""The 64-bit container (CUCM_FORMAT_64), checked on the host.

Its chunk payloads are the reference's; only the framing widens: a 45-byte
header (ff ff ff ff 00 00 00 02, then 64-bit sizes) and 8-byte batch sizes and
chunk end offsets.  The host framing (cucm_frame_bodies) writes it from the
oracle's batch bodies; the payloads it frames must be the ones the 32-bit
container holds, and the size query must read the 64-bit size.
"""
import ctypes
import struct

import pytest

import cucm_b200 as cc
from cucm_b200 import workloads as W


def _payloads32(blob, cs):
    """Chunk payloads of a reference container without prelearn."""
    n = struct.unpack(">I", blob[:4])[0]
    nch = (n + cs - 1) // cs
    batch = struct.unpack(">H", blob[4:6])[0]
    out, pos = [], 21
    for k0 in range(0, nch, batch):
        C = min(batch, nch - k0)
        bsz = struct.unpack("<I", blob[pos:pos + 4])[0]
        body = blob[pos + 4:pos + 4 + bsz]
        ends = [struct.unpack(">I", body[4 * i:4 * i + 4])[0] + 1 - 4 * C for i in range(C)]
        start = 0
        for e in ends:
            out.append(body[4 * C + start:4 * C + e])
            start = e
        pos += 4 + bsz
    return out


def _payloads64(blob):
    assert blob[:8] == b"\xff\xff\xff\xff\x00\x00\x00\x02"
    n, batch, unit, cs, coded, raw = struct.unpack(">QIIIQQ", blob[8:44])
    assert coded == 0 and raw == 0 and blob[44] == 0
    nch = (n + cs - 1) // cs
    out, pos = [], 45
    for k0 in range(0, nch, batch):
        C = min(batch, nch - k0)
        bsz = struct.unpack("<Q", blob[pos:pos + 8])[0]
        body = blob[pos + 8:pos + 8 + bsz]
        ends = [struct.unpack(">Q", body[8 * i:8 * i + 8])[0] + 1 - 8 * C for i in range(C)]
        start = 0
        for e in ends:
            out.append(body[8 * C + start:8 * C + e])
            start = e
        pos += 8 + bsz
    assert pos == len(blob)
    return n, batch, unit, cs, out


@pytest.mark.parametrize("size,cs,batch", [(40000, 4096, 3), (8192, 4096, 100), (5000, 4096, 1)])
def test_frame64_holds_the_reference_payloads(oracle_mod, cucm_lib, size, cs, batch):
    data = W.text(size, size).tobytes()
    v1 = oracle_mod.compress(data, cs, 128, 0, batch)
    body = oracle_mod.compress(data, cs, 128, 0, 65535)[25:]
    nch = (size + cs - 1) // cs
    assert cc.frame_bodies([body], [nch], size, cs, 128, batch) == v1
    v2 = cc.frame_bodies([body], [nch], size, cs, 128, batch, fmt=cc.FORMAT_64)
    n, b, u, c, pays = _payloads64(v2)
    assert (n, b, u, c) == (size, batch, 128, cs)
    assert pays == _payloads32(v1, cs)
    got = ctypes.c_uint64()
    assert cucm_lib.cucm_decompressed_size(v2, len(v2), ctypes.byref(got)) == 0 and got.value == size
    # a 32-bit header with the batch count 0 is not a container
    bad = b"\xff\xff\xff\xff\x00\x00\x00\x03" + v2[8:]
    h = ctypes.c_void_p()
    assert cucm_lib.cucm_model_from_container(bad, len(bad), ctypes.byref(h)) == -3


def test_format_field_checks(cucm_lib):
    p = cc.default_params(chunksize=4096)
    assert p.format == cc.FORMAT_AUTO
    # the 32-bit container cannot hold more than 4 GiB of input
    p32 = cc.default_params(chunksize=1 << 20, fmt=cc.FORMAT_32)
    p64 = cc.default_params(chunksize=1 << 20, fmt=cc.FORMAT_64)
    pa = cc.default_params(chunksize=1 << 20)
    big = (5 << 30)
    assert cucm_lib.cucm_compress_bound(big, ctypes.byref(pa)) == cucm_lib.cucm_compress_bound(big, ctypes.byref(p64))
    assert cucm_lib.cucm_compress_bound(100, ctypes.byref(p64)) > cucm_lib.cucm_compress_bound(100, ctypes.byref(p32))
    out = ctypes.create_string_buffer(64)
    got = ctypes.c_uint64()
    p32.chunksize = 4096
    bad = cc.default_params(chunksize=4096, fmt=7)
    assert cucm_lib.cucm_frame_bodies(ctypes.byref(bad), 0, 0, None, None, None, out, 64, ctypes.byref(got)) == -1
    assert cucm_lib.cucm_frame_bodies(ctypes.byref(p32), 0, 0, None, None, None, out, 64, ctypes.byref(got)) == 0
    assert got.value == 21
    p64.chunksize = 4096
    assert cucm_lib.cucm_frame_bodies(ctypes.byref(p64), 0, 0, None, None, None, out, 64, ctypes.byref(got)) == 0
    assert got.value == 45 and out.raw[:8] == b"\xff\xff\xff\xff\x00\x00\x00\x02"
