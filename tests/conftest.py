import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a) and the built libpawan_gpu.so")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def ref_available():
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("oracle/_ref/libpawanref.so is not built (make -C oracle)")
    return True


@pytest.fixture(scope="session")
def ref_ho_available():
    from oracle import oracle as O
    if not O.ref_available("highorder"):
        pytest.skip("oracle/_ref/libpawanref_ho.so is not built (make -C oracle)")
    return True


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a visible CUDA device")
    from pawan_b200 import capi
    capi.load()
    return True
