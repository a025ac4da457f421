import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def kpzb():
    """The product package; importing it loads libkpzb200.so (no fallback)."""
    import cudakpz_b200
    return cudakpz_b200


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    return o
