import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def oracle():
    from oracle import bindings
    return bindings.port()


@pytest.fixture(scope="session")
def ref_lib():
    from oracle import bindings
    lib = bindings.reference()
    if lib is None:
        pytest.skip("oracle/_ref/libencore_ref.so not built (needs the reference sources)")
    return lib


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
