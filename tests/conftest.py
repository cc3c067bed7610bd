import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "reference: needs the reference tree compiled into oracle/_ref")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds (or refreshes) the native libraries once per session."""
    from disco_b200 import build as B
    B.build(verbose=False)
    from oracle import build_oracle
    build_oracle.build(verbose=False)
    yield


def has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
