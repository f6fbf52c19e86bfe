import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "dress-graph_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: larger parity case")


@pytest.fixture(scope="session")
def oracle_port():
    import oracle
    return oracle.port()


@pytest.fixture(scope="session")
def oracle_ref():
    import oracle
    r = oracle.reference()
    if r is None:
        pytest.skip("reference library not built (oracle/_ref)")
    return r
