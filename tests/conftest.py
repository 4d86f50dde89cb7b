"""Shared fixtures.  `-m gpu` tests need a B200 and the built extension;
everything else runs on CPU.  The oracle (oracle/) is the checker only."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libhercules_gpu.so")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.build(ref=False)
    return O


@pytest.fixture(scope="session")
def hg():
    import hercules_b200 as H
    from hercules_b200 import build as B
    B.build()
    H.lib()
    return H


@pytest.fixture(scope="session")
def gpu_available():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


def golden_path(name):
    return os.path.join(ROOT, "tests", "golden", name)
