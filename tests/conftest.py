import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "llg-sim_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.lib()
    oracle.set_threads(min(8, os.cpu_count() or 1))
    return oracle


@pytest.fixture(scope="session")
def gpu():
    import llg_b200

    llg_b200.lib()
    return llg_b200
