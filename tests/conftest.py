"""pytest configuration: the `gpu` marker and shared fixtures.

GPU tests call the product through its C ABI (libcuopus.so) and compare with
the oracle (oracle/: libopus 1.5.2 fixed point built from the reference's
vendored sources, and the CPU restatements).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libcuopus.so")


@pytest.fixture(scope="session")
def root():
    return ROOT


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch
