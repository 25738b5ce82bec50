import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    """The reference's own CPU code (oracle/_ref), when it was built."""
    from oracle import REF_SO, Reference, build_reference
    if not os.path.exists(REF_SO) and not build_reference():
        pytest.skip("reference CPU build unavailable (no reference tree at build time)")
    return Reference()
