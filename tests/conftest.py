import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    """Skip-free GPU gate: -m gpu tests fail loudly when no device is visible."""
    if not _cuda_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    import torch
    torch.cuda.init()
    return torch.device("cuda:0")
