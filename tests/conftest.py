import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "iron-array_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ia():
    """The C-ABI binding, initialised on the GPU (fails loudly without one)."""
    import iarray_b200 as m
    m.init()
    return m


@pytest.fixture(scope="session")
def ctx(ia):
    c = ia.Context()
    yield c
    c.close()
