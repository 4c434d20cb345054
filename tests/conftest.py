"""Shared fixtures.  Tests marked ``gpu`` need a B200 and the built libcoulktt.so;
everything else runs on a CPU-only host."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU and the built CUDA library")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def ctx():
    import ktt_b200
    c = ktt_b200.CoulombContext(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(REPO, "tests", "golden")
