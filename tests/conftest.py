"""Shared test setup: import paths, the `gpu` marker and device fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "indigenous-cpu-gpu-optimization-engine-for-indian-industry_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def hn():
    """The sm_100a library, initialised on device 0 (fails loudly if absent)."""
    import torch

    import hnb200

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    torch.cuda.set_device(0)
    torch.zeros(1, device="cuda")  # torch's context first: both share the primary context
    hnb200.init(0)
    return hnb200


@pytest.fixture(scope="session")
def torch_cuda(hn):
    import torch

    return torch
