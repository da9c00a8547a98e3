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
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) and the built liboxb200.so")


@pytest.fixture(scope="session")
def backend():
    from oxidelake_b200.backend import CudaBackend

    return CudaBackend(int(os.environ.get("OXB200_DEVICE", "0")))


@pytest.fixture(scope="session")
def stream(backend):
    return backend.create_stream()
