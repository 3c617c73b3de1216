import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100) and libcucm.so")


@pytest.fixture(scope="session")
def cucm_lib():
    """The built C-ABI library (built in-tree if missing)."""
    from cucm_b200 import build as b
    b.build()
    import cucm_b200
    return cucm_b200.lib()


@pytest.fixture(scope="session")
def oracle_mod():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "libcucm_oracle.so", "oracle_cli"],
                   check=True)
    import oracle
    return oracle


@pytest.fixture(scope="session")
def gpu_ctx(cucm_lib):
    """A context on cuda:0; fails loudly if the device or library is unusable."""
    import cucm_b200
    ctx = cucm_b200.Context(0)
    yield ctx
    ctx.close()
