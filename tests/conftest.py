import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and liblepic_gpu.so")
    config.addinivalue_line("markers", "slow: long-running test")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    oracle.set_threads(1)
    return oracle


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
