import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library; GPU tests fail (not skip) when it cannot be loaded
    on a machine that has a GPU."""
    from medyan_b200 import lib
    if not _cuda_available():
        pytest.skip("no CUDA device")
    return lib.load()
