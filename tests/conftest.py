"""pytest configuration: the ``gpu`` marker and shared fixtures.

``-m "not gpu"`` runs on any machine (oracle vs golden fixtures, oracle vs
the compiled reference, host logic, library loading); ``-m gpu`` runs the
parity tests of the CUDA kernels on a B200 through the C ABI.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size workloads (seconds to minutes)")


@pytest.fixture(scope="session")
def golden():
    path = os.path.join(ROOT, "tests", "golden", "golden.npz")
    return np.load(path, allow_pickle=False)


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu-marked tests")
    return torch.device("cuda:0")
