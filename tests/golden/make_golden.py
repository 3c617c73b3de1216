#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ with the reference's own code.

The reference ships no test vectors, so the fixtures are produced by running
the reference itself: oracle/_ref/cucm_compress_ref and
oracle/_ref/cucm_decompress_ref, built from the reference's unmodified
sources by oracle/make_ref.py (run `make -C oracle ref` first, in a checkout
that has the reference sources).

For every case the inputs are regenerated from a seed (see CASES), so only
the reference's outputs are stored: <name>.cucm (the container the
reference's compressor wrote) and a manifest entry with the parameters and
SHA-256 of input and output.  The reference decompressor is also run on each
container and must reproduce the input.

Usage:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.golden.golden_inputs import CASES, make_input  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")


def sha(b):
    return hashlib.sha256(b).hexdigest()


def main():
    comp = os.path.join(REF, "cucm_compress_ref")
    decomp = os.path.join(REF, "cucm_decompress_ref")
    if not (os.path.exists(comp) and os.path.exists(decomp)):
        sys.exit("reference binaries missing; run `make -C oracle ref`")
    manifest = []
    with tempfile.TemporaryDirectory() as tmp:
        for case in CASES:
            data = make_input(case)
            src = os.path.join(tmp, "in.bin")
            dst = os.path.join(tmp, "out.cucm")
            back = os.path.join(tmp, "back.bin")
            with open(src, "wb") as f:
                f.write(data)
            cmd = [comp, "-f", src, "-o", dst, "-s", str(case["chunksize"]), "-u", str(case["unit"]),
                   "-b", str(case["batch"])]
            if case["prelearn"]:
                cmd += ["-p", str(case["prelearn"])]
            subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
            with open(dst, "rb") as f:
                blob = f.read()
            subprocess.run([decomp, "-i", dst, "-o", back], check=True, stdout=subprocess.DEVNULL)
            with open(back, "rb") as f:
                assert f.read() == data, "reference round trip failed for %s" % case["name"]
            with open(os.path.join(HERE, case["name"] + ".cucm"), "wb") as f:
                f.write(blob)
            entry = dict(case)
            entry.update(input_sha256=sha(data), input_len=len(data), output_sha256=sha(blob),
                         output_len=len(blob))
            manifest.append(entry)
            print("%-24s %8d -> %8d" % (case["name"], len(data), len(blob)))
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
