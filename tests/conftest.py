"""Shared test setup: import paths, the gpu marker, and small helpers."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "hsi-detectors-cuda_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden", "golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN, allow_pickle=False)


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.fp64_lib()
    return oracle


@pytest.fixture(scope="session")
def hsi():
    """The product binding; GPU tests fail loudly if the library or device is missing."""
    import torch
    import hsi_b200
    if not torch.cuda.is_available():
        pytest.fail("gpu test run without a CUDA device")
    hsi_b200.lib()
    return hsi_b200
