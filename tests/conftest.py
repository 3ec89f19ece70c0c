import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

REF_ROOT = "/root/reference"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    """The oracle module with its restatement built (and the reference, where
    its sources are present; on a machine without them the prebuilt
    oracle/_ref library is used if it travelled with the tree)."""
    import oracle as O

    if not os.path.exists(O.LIB_ORACLE):
        O.build(ref_root="/nonexistent")
    if not os.path.exists(O.LIB_REF) and os.path.isdir(os.path.join(REF_ROOT, "src")):
        O.build(ref_root=REF_ROOT)
    return O


@pytest.fixture(scope="session")
def psi():
    from pypsi_b200 import PSI

    return PSI


@pytest.fixture(scope="session")
def gpu(psi):
    if psi.device_count() <= 0:
        pytest.fail("GPU test run without a visible CUDA device")
    return psi
