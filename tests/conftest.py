import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)



def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session", autouse=True)
def built():
    """Build libbbpd and the oracle if they are missing (no-op when prebuilt)."""
    from bb_pd_b200 import build as b
    lib = os.path.join(ROOT, "bb_pd_b200", "lib", "libbbpd.so")
    if not os.path.exists(lib):
        b.build()
    # oracle/Makefile decides what is stale; it builds the reference routines
    # only where the reference tree exists (the build machine), and the
    # prebuilt oracle/_ref travels with the tree everywhere else
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libbbpd_ref.so")) or \
            not os.path.exists(os.path.join(ROOT, "oracle", "_build", "liboracle.so")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-s"], check=True)
    yield
