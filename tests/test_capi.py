"""Host-side checks of the C ABI that need no GPU: the library loads,
exports every entry point that include/cucm.h declares, validates arguments
and parses container headers."""
import ctypes
import os
import re

import pytest

import cucm_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "cucm.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(cucm_\w+)\s*\(", text)))


def test_header_and_binding_agree(cucm_lib):
    declared = _declared()
    bound = sorted(n for n, _, _ in cucm_b200.SIGNATURES)
    assert declared == bound


def test_library_exports_all_symbols(cucm_lib):
    for name in _declared():
        assert hasattr(cucm_lib, name), name


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_ctx_create_without_gpu_fails_loudly(cucm_lib):
    h = ctypes.c_void_p()
    assert cucm_lib.cucm_ctx_create(0, None, ctypes.byref(h)) == -6  # CUCM_ENODEV
    with pytest.raises(cucm_b200.CucmError):
        cucm_b200.Context(0)
    assert cucm_lib.cucm_server_create(0, 0, None, ctypes.byref(h)) == -6
    with pytest.raises(cucm_b200.CucmError):
        cucm_b200.Server(0)


def test_serve_calls_reject_bad_arguments(cucm_lib):
    rid = ctypes.c_uint64()
    assert cucm_lib.cucm_serve_submit(None, 0, None, 0, None, None, 0, ctypes.byref(rid)) == -1
    assert cucm_lib.cucm_serve_poll(None, 1, 0, None, None, None) == -1
    assert cucm_lib.cucm_server_destroy(None) == -1
    assert cucm_lib.cucm_server_set_queue_limit(None, 4) == -1


def test_default_params_match_reference_cli(cucm_lib):
    p = cucm_b200.default_params()
    assert (p.chunksize, p.unit, p.prelearn, p.batch) == (1 << 20, 128, 0, 100)


def test_compress_bound_and_size_query(cucm_lib):
    p = cucm_b200.default_params(chunksize=4096)
    assert cucm_lib.cucm_compress_bound(0, ctypes.byref(p)) == 21 + 8
    assert cucm_lib.cucm_compress_bound(10000, ctypes.byref(p)) >= 3 * (32 * 4096 + 5)
    hdr = bytes([0, 1, 0, 0]) + bytes(17)
    size = ctypes.c_uint64()
    assert cucm_lib.cucm_decompressed_size(hdr, len(hdr), ctypes.byref(size)) == 0
    assert size.value == 65536
    assert cucm_lib.cucm_decompressed_size(hdr, 3, ctypes.byref(size)) == -3


def test_strerror(cucm_lib):
    for s in range(0, -11, -1):
        assert cucm_lib.cucm_strerror(s)
    assert b"different bytes" in cucm_lib.cucm_strerror(cucm_b200.EMISMATCH)


def test_tuning_layout_and_autotune_arguments(cucm_lib):
    # cucm_tuning: form, spec_bits, max_slots, (pad), hbm_budget, kernel, dec_pairs, dec_tables, cmp_ctas,
    # dec_spin_limit, (pad)
    assert ctypes.sizeof(cucm_b200.Tuning) == 48
    assert (cucm_b200.Tuning.dec_tables.offset, cucm_b200.Tuning.cmp_ctas.offset) == (32, 36)
    assert cucm_b200.Tuning.dec_spin_limit.offset == 40
    assert cucm_lib.cucm_ctx_get_tuning(None, None) == -1
    t = cucm_b200.Tuning()
    p = cucm_b200.default_params()
    n = ctypes.c_uint32()
    buf = ctypes.create_string_buffer(16)
    assert cucm_lib.cucm_autotune(None, buf, 16, ctypes.byref(p), 1, None, 0, ctypes.byref(n), ctypes.byref(t)) == -1
    # a null result array with a nonzero capacity is refused before any device work
    assert cucm_lib.cucm_autotune(None, buf, 16, ctypes.byref(p), 1, None, 4, ctypes.byref(n), ctypes.byref(t)) == -1


def test_model_from_container_host_side(cucm_lib):
    """The prelearn model is host work (no GPU): a container without a
    prelearn block has no model, a malformed header is refused."""
    gold = os.path.join(ROOT, "tests", "golden")
    with open(os.path.join(gold, "text_20k_cs4k.cucm"), "rb") as f:
        plain = f.read()
    h = ctypes.c_void_p()
    assert cucm_lib.cucm_model_from_container(plain, len(plain), ctypes.byref(h)) == 0 and not h.value
    assert cucm_lib.cucm_model_from_container(plain, 10, ctypes.byref(h)) == -3
    assert cucm_lib.cucm_model_destroy(None) == -1
    with open(os.path.join(gold, "text_12k_pre3000.cucm"), "rb") as f:
        pre = f.read()
    m = cucm_b200.Model.from_container(pre)
    assert m is not None
    m.close()
    m = cucm_b200.Model.prelearn(b"some prefix bytes" * 10)
    m.close()


def test_frame_bodies_argument_checks(cucm_lib):
    p = cucm_b200.default_params(chunksize=4096)
    got = ctypes.c_uint64()
    # chunk counts that do not add up to the stream's chunks
    body = (ctypes.c_void_p * 1)(None)
    ns = (ctypes.c_uint64 * 1)(0)
    cs = (ctypes.c_uint32 * 1)(2)
    assert cucm_lib.cucm_frame_bodies(ctypes.byref(p), 4096, 1, body, ns, cs, None, 0, ctypes.byref(got)) == -1
    # the empty stream: header only
    out = ctypes.create_string_buffer(64)
    assert cucm_lib.cucm_frame_bodies(ctypes.byref(p), 0, 0, None, None, None, out, 64, ctypes.byref(got)) == 0
    assert got.value == 21
