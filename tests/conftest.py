import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long CPU case")


@pytest.fixture(scope="session")
def oracle():
    from oracle_py import Oracle  # noqa: F401  (builds on first use)
    import oracle_py
    oracle_py.ensure_built()
    return oracle_py
