import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests" / "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def _build_library():
    from cubie_b200 import _native
    _native.build_library()
    yield


@pytest.fixture(scope="session")
def cuda_device():
    if not gpu_available():
        pytest.fail("this test needs a CUDA GPU; run the CPU suite with -m 'not gpu'")
    return 0
