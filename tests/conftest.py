import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def engine():
    """The B200 engine package (its directory name is not an identifier)."""
    return importlib.import_module("1_b200")


@pytest.fixture(scope="session")
def eng():
    return engine()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch


REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libgpukern_ref.so")
