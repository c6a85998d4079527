import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session")
def gpu():
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    import graphblas_b200 as gb
    gb.init()
    return gb


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()
