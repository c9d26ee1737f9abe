import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


_HAS_GPU = None


def has_gpu() -> bool:
    global _HAS_GPU
    if _HAS_GPU is None:
        try:
            import torch
            _HAS_GPU = bool(torch.cuda.is_available())
        except Exception:
            _HAS_GPU = False
    return _HAS_GPU


@pytest.fixture
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    return True
