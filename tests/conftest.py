import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libflursys_cuda.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import binding
    binding.build()
    binding.load()
    binding.set_threads(1)
    return binding


@pytest.fixture(scope="session")
def cudalib():
    from flursys_b200 import _abi
    return _abi.load()
