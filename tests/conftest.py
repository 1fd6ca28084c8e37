import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: long-running")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    return True


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the CUDA libraries (nvcc cross-compiles without a GPU) and the oracle once."""
    from irs_b200 import build
    build.build(jobs=4)
    from oracle import pyoracle
    pyoracle.build()
