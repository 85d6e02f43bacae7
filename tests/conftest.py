import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "xblossom-sigmetrics27-ae_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds libxbtrav.so and the oracle if they are missing or stale."""
    import build_lib
    from oracle import oracle

    build_lib.build()
    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build()
    yield


@pytest.fixture(scope="session")
def ctx():
    import xbtrav

    c = xbtrav.Context(0)
    yield c
    c.close()
