"""The fixed-model variant (the paper's section 4.5), on the host.

The reference ships no code for it, so the oracle's restatement
(co_compress_ex with fixed = 1: the prelearned model codes every chunk's data
bits, never updated) defines its stream; parity for it is against that
restatement only.  Here: the oracle's own round trip, the header flag, and
the library's host-side checks of the parameters.
"""
import ctypes

import pytest

import cucm_b200 as cc
from cucm_b200 import workloads as W


@pytest.mark.parametrize("size,cs,pre", [(60000, 16384, 8000), (20000, 65536, 3000), (5000, 4096, 4096)])
def test_oracle_fixed_round_trip(oracle_mod, size, cs, pre):
    data = W.text(size, size).tobytes()
    blob = oracle_mod.compress(data, cs, 128, pre, 100, fixed=True)
    assert blob[20] & 2
    assert oracle_mod.decompress(blob) == data
    # the adaptive stream of the same input differs only in its payloads and flag
    ad = oracle_mod.compress(data, cs, 128, pre, 100)
    assert ad[:20] == blob[:20] and ad[20] | 2 == blob[20]


def test_fixed_needs_prelearn(cucm_lib, oracle_mod):
    with pytest.raises(RuntimeError):
        oracle_mod.compress(b"x" * 1000, 4096, 128, 0, 100, fixed=True)
    p = cc.default_params(chunksize=4096, fixed=True)
    out = ctypes.create_string_buffer(64)
    got = ctypes.c_uint64()
    # frame_bodies refuses it (and any prelearn): the variant is not a reference stream
    assert cucm_lib.cucm_frame_bodies(ctypes.byref(p), 0, 0, None, None, None, out, 64, ctypes.byref(got)) == -1


def test_fixed_container_model_readable(cucm_lib, oracle_mod):
    data = W.text(30000, 7).tobytes()
    blob = oracle_mod.compress(data, 8192, 128, 5000, 100, fixed=True)
    m = cc.Model.from_container(blob)
    assert m is not None
    m.close()
    bad = bytearray(blob)
    bad[20] = 7  # unknown flag bits
    h = ctypes.c_void_p()
    assert cucm_lib.cucm_model_from_container(bytes(bad), len(bad), ctypes.byref(h)) == -3
