import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the product path")


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def built():
    """Builds libmpf.so and the oracle once per session (no-op when up to date)."""
    from mapol_b200 import build

    build.build()
    return True


@pytest.fixture(scope="session")
def gpu(built):
    if not _has_gpu():
        pytest.skip("no CUDA device")
    return True
