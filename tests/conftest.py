import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU case")


@pytest.fixture(scope="session")
def ctx():
    """A vaco_av1 context on cuda:0 (GPU tests only)."""
    from vaco_b200.gpu import Context

    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def oracle_threads():
    return max(1, min(32, os.cpu_count() or 1))
