import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libmcm_gpu.so")
    config.addinivalue_line("markers", "slow: longer CPU test")


def have_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_lib():
    if not have_gpu():
        pytest.skip("no CUDA device")
    from mcmtop_b200 import _abi

    return _abi.load()


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import pyoracle

    return pyoracle.load()
