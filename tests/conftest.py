import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build(ref=True)
    return oracle


@pytest.fixture(scope="session")
def ucg():
    """The product library; built in-tree if stale (nvcc cross-compiles)."""
    from unicycle_b200 import build
    build.build()
    import unicycle_b200
    unicycle_b200.load()
    return unicycle_b200
