import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "diff-triangle-tracer_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle

    if not pyoracle.oracle_available():
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "lib"], check=True)
    o = pyoracle.Oracle()
    yield o
    o.close()


@pytest.fixture(scope="session")
def reference():
    from oracle import pyoracle

    if not pyoracle.reference_available():
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref-if-present"], check=True)
    if not pyoracle.reference_available():
        pytest.skip("host build of the reference's sources is not available")
    r = pyoracle.Reference()
    yield r
    r.close()
