import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REF_TREE = "/root/reference"   # present only on the build machine; never needed at run time


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
    if not os.path.exists(os.path.join(ROOT, "oracle", "_build", "liboracle.so")) or (
            os.path.isdir(REF_TREE) and not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libbbpd_ref.so"))):
        args = ["make", "-C", os.path.join(ROOT, "oracle"), "-s"]
        if os.path.isdir(REF_TREE):
            args.append(f"REF={REF_TREE}")
        subprocess.run(args, check=True)
    yield
