"""The drop-in CLIs end to end on the GPU.

`cucm_compress -f IN -o OUT -s -u -b [-p]` must write the reference's
container byte for byte (the golden fixtures are the reference's own output)
and print the reference's result lines (cucm_compress_v2.cu:1411-1415);
`cucm_decompress -i OUT -o BACK -a 3` must give the input back and print the
reference's finish line (cucm_decompress_v2.cu:1306-1308).  Where the
reference's host build is present (oracle/_ref), its printed size and ratio
lines are compared with ours for the same flags.
"""
import json
import os
import re
import subprocess

import pytest

from tests.golden.golden_inputs import make_input

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cucm_b200", "bin")
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF = os.path.join(ROOT, "oracle", "_ref", "cucm_compress_ref")
with open(os.path.join(GOLDEN, "manifest.json")) as _f:
    MANIFEST = {e["name"]: e for e in json.load(_f)}

NAMES = ["text_20k_cs4k", "text_20k_cs4k_b2", "text_12k_pre3000", "random_12k_pre2000", "text_10k_u32",
         "text_4097_cs4096_u64", "text_0_cs4k", "text_9_cs8"]
# cases also run through the reference's host build (it allocates 256 MiB of
# tables per chunk, so only a few)
WITH_REF = {"text_20k_cs4k_b2", "text_12k_pre3000", "text_0_cs4k"}


def _size_arg(v):
    """The CLI's size syntax: K/M suffixes where they divide evenly."""
    for suffix, mult in (("M", 1 << 20), ("K", 1 << 10)):
        if v and v % mult == 0:
            return "%d%s" % (v // mult, suffix)
    return str(v)


def _result_lines(text):
    keep = ("Original size", "Compressed size", "Compression ratio")
    return [ln for ln in text.splitlines() if ln.startswith(keep)]


@pytest.mark.parametrize("name", NAMES)
def test_cli_matches_golden(cucm_lib, tmp_path, name):
    e = MANIFEST[name]
    data = make_input(e)
    src, dst, back = tmp_path / "in.bin", tmp_path / "out.cucm", tmp_path / "back.bin"
    src.write_bytes(data)
    flags = ["-s", _size_arg(e["chunksize"]), "-u", str(e["unit"]), "-b", str(e["batch"])]
    if e["prelearn"]:
        flags += ["-p", _size_arg(e["prelearn"])]
    r = subprocess.run([os.path.join(BIN, "cucm_compress"), "-f", str(src), "-o", str(dst)] + flags,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    with open(os.path.join(GOLDEN, name + ".cucm"), "rb") as f:
        golden = f.read()
    assert dst.read_bytes() == golden
    lines = _result_lines(r.stdout)
    assert lines[0] == "Original size  : %d bytes" % len(data)
    nchunks = -(-(len(data) - e["prelearn"]) // e["chunksize"])
    nbatches = -(-nchunks // e["batch"])
    assert lines[1] == "Compressed size: %d bytes" % (len(golden) - 4 * nbatches)
    assert lines[2].startswith("Compression ratio: ")
    if name in WITH_REF and os.path.exists(REF):
        ref_out = tmp_path / "ref.cucm"
        rr = subprocess.run([REF, "-f", str(src), "-o", str(ref_out)] + flags, capture_output=True, text=True)
        assert rr.returncode == 0
        assert _result_lines(rr.stdout) == lines
        assert ref_out.read_bytes() == golden
    r = subprocess.run([os.path.join(BIN, "cucm_decompress"), "-i", str(dst), "-o", str(back), "-a", "3"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert back.read_bytes() == data
    assert re.search(r"^Decompression finished: %s -> %s \(%d bytes, maxassumed_length=3\)$"
                     % (re.escape(str(dst)), re.escape(str(back)), len(data)), r.stdout, re.M)


def test_cli_chunknum_truncates(cucm_lib, tmp_path, oracle_mod):
    """-c N keeps the first N chunks, as the reference's main does
    (cucm_compress_v2.cu:1398-1400)."""
    data = make_input(dict(kind="text", size=30000, seed=12))
    src, dst = tmp_path / "in.bin", tmp_path / "out.cucm"
    src.write_bytes(data)
    r = subprocess.run([os.path.join(BIN, "cucm_compress"), "-f", str(src), "-o", str(dst), "-s", "4K", "-c", "3"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert dst.read_bytes() == oracle_mod.compress(data[:3 * 4096], 4096, 128, 0, 100)
