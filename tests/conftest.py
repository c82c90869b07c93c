import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ref():
    """The reference CPU build (oracle/_ref), or skip when it was not built."""
    from oracle import ref as R
    if not R.available():
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    return R
