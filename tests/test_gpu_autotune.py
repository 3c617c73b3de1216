"""The measured autotuner (cucm_autotune): every execution choice it tries
must give the same container and give the sample back, and the choice it
applies is the fastest it measured.  The knobs it turns -- launch form,
compressor CTAs per SM, warps per chunk (pipelined or generic kernels),
decoder chunks per CTA, order 0/1 table placement -- never change a byte."""
import pytest

import cucm_b200 as cc
from cucm_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture
def ctx(gpu_ctx):
    """The session's context, its default tuning restored afterwards."""
    yield gpu_ctx
    gpu_ctx.set_tuning()


def test_autotune_measures_every_choice_and_applies_the_fastest(ctx, oracle_mod):
    sample = W.make("text", 300000, 11).tobytes() + W.make("walk", 200000, 12).tobytes()
    want = oracle_mod.compress(sample, 16384, 128, 0, 100)
    best, cands = ctx.autotune(sample, reps=1, chunksize=16384)
    comp_c = [c for c in cands if c["compress_ms"] >= 0]
    dec_c = [c for c in cands if c["decompress_ms"] >= 0]
    # compressor: persistent with 1 or 2 CTAs per SM, plain, persistent
    # generic (8 warps per chunk); decoder: persistent with 0..5 chunks per
    # CTA x 2 table placements, plain x 2, persistent generic
    assert (len(comp_c), len(dec_c)) == (4, 15)
    assert sum(c["kernel"] == 1 for c in comp_c) == 1 and sum(c["kernel"] == 1 for c in dec_c) == 1
    assert all(c["compress_ms"] > 0 for c in comp_c) and all(c["decompress_ms"] > 0 for c in dec_c)
    totals = {}
    for form in (cc.FORM_PERSISTENT, cc.FORM_PLAIN):
        for kern in (0, 1):
            cs = [c for c in comp_c if c["form"] == form and c["kernel"] == kern]
            ds = [c for c in dec_c if c["form"] == form and c["kernel"] == kern]
            if not cs or not ds:
                continue
            bc = min(cs, key=lambda c: c["compress_ms"])
            bd = min(ds, key=lambda c: c["decompress_ms"])
            totals[(form, kern)] = (bc["compress_ms"] + bd["decompress_ms"], bc["cmp_ctas"], bd["dec_pairs"],
                                    bd["dec_tables"])
    form, kern = min(totals, key=lambda f: totals[f][0])
    assert ((best["form"], best["kernel"], best["cmp_ctas"], best["dec_pairs"], best["dec_tables"])
            == (form, kern) + totals[(form, kern)][1:])
    assert ctx.get_tuning() == best
    comp = ctx.compress(sample, chunksize=16384)
    assert comp == want
    assert ctx.decompress(comp) == sample


@pytest.mark.parametrize("cmp_ctas", [1, 2])
def test_compressor_ctas_per_sm_keep_the_bytes(ctx, oracle_mod, cmp_ctas):
    buf = W.make("walk", 120000, 31).tobytes()
    ctx.set_tuning(form=cc.FORM_PERSISTENT, cmp_ctas=cmp_ctas)
    assert ctx.compress(buf, chunksize=4096) == oracle_mod.compress(buf, 4096, 128, 0, 100)


@pytest.mark.parametrize("dec_pairs,dec_tables", [(1, 0), (1, 1), (2, 0), (3, 1), (5, 1)])
def test_decoder_knobs_keep_the_bytes(ctx, oracle_mod, dec_pairs, dec_tables):
    buf = W.make("text", 150000, 21).tobytes()
    comp = oracle_mod.compress(buf, 8192, 128, 0, 100)
    ctx.set_tuning(form=cc.FORM_PERSISTENT, dec_pairs=dec_pairs, dec_tables=dec_tables)
    assert ctx.decompress(comp) == buf
    assert ctx.compress(buf, chunksize=8192) == comp
