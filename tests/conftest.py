import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a); runs through the C ABI")


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device for gpu-marked tests; fails (does not skip) when none is present."""
    import torch
    assert torch.cuda.is_available(), "gpu-marked test needs a CUDA device"
    torch.cuda.init()
    return torch.device("cuda:0")
