"""Test configuration: import paths and the `gpu` marker.

`-m "not gpu"` runs the CPU suite (oracle vs the reference's known answers,
host logic, C-ABI load/export checks). `-m gpu` runs the parity tests of the
CUDA path on an sm_100 device; they call libskgemm through its C ABI.
"""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "stream-k-gemm_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU and the built libskgemm.so")
    config.addinivalue_line("markers", "slow: long-running (full-size configurations)")


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return dict(np.load(os.path.join(REPO, "tests", "golden", "reference_known_answers.npz")))


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return torch.device("cuda:0")
