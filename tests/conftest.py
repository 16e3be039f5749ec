import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "planktonindividuals.jl_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libpib200.so")
    config.addinivalue_line("markers", "slow: long-running")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_lib():
    if not has_gpu():
        pytest.fail("GPU test without a CUDA device: run the gpu-marked tests on a B200")
    import build as _b  # planktonindividuals.jl_b200/build.py
    _b.build()
    from PlanktonIndividuals import _lib
    return _lib.load()
