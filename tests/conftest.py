import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
TESTS = Path(__file__).resolve().parent
if str(TESTS) not in sys.path:
    sys.path.insert(0, str(TESTS))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def golden_dir():
    return TESTS / "golden"


@pytest.fixture(scope="session", autouse=True)
def _product_library_built():
    """Builds libsigmo_b200.so (nvcc, sm_100a) when a fresh checkout lacks it;
    the oracle's library builds itself on first use."""
    from sigmo_b200 import _lib

    if not _lib.LIB_PATH.exists():
        from sigmo_b200 import build

        build.build()
