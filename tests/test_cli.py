"""Flag handling of the drop-in CLIs that needs no GPU (cucm_compress_v2.cu:
1301-1418, cucm_decompress_v2.cu:1258-1314)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cucm_b200", "bin")


def run(*args):
    return subprocess.run(list(args), capture_output=True, text=True)


@pytest.fixture(scope="module")
def bins(cucm_lib):
    return os.path.join(BIN, "cucm_compress"), os.path.join(BIN, "cucm_decompress")


def test_compress_help(bins):
    r = run(bins[0])
    assert r.returncode == 0 and "Usage" in r.stdout
    r = run(bins[0], "-h")
    assert r.returncode == 0 and "--chunksize" in r.stdout


@pytest.mark.parametrize("args", [["-u", "48"], ["-u", "100"], ["-u", "0"], ["-s", "abc"], ["-b", "0"],
                                  ["-c", "0"], ["--bogus"]])
def test_compress_rejects(bins, args, tmp_path):
    r = run(bins[0], *args, "-f", str(tmp_path / "none"))
    assert r.returncode == 1


def test_compress_missing_input(bins, tmp_path):
    r = run(bins[0], "-f", str(tmp_path / "missing.bin"), "-o", str(tmp_path / "o"))
    assert r.returncode == 1 and "Failed to open input file" in r.stderr


def test_decompress_usage(bins, tmp_path):
    assert run(bins[1]).returncode == 1
    assert run(bins[1], "-i", "x").returncode == 1
    assert run(bins[1], "-x").returncode == 1
    r = run(bins[1], "-i", str(tmp_path / "missing"), "-o", str(tmp_path / "o"))
    assert r.returncode == 1
