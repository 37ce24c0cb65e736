import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: large parity case")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import build_oracle, oracle
    build_oracle.build()
    return oracle
