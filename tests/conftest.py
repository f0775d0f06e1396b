import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


def oracle_available():
    return os.path.exists(os.path.join(ROOT, "oracle", "_ref", "liboracle.so")) or os.path.isdir("/root/reference")


@pytest.fixture(scope="session")
def oracle_mod():
    if not oracle_available():
        pytest.skip("oracle library not built")
    from oracle import oracle
    return oracle
