"""Test configuration: the `gpu` marker, and one-time builds of the checker
(oracle/) and of the product library when they are missing."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    from oracle import oracle as O
    if not os.path.exists(O.LIB_PATH):
        O.build()
    import madmax_b200.build as B
    if not os.path.exists(B.LIB):
        B.build()
    yield


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(ROOT, "tests", "golden")
