import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C-ABI")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def pytest_collection_modifyitems(config, items):
    # GPU tests fail loudly rather than skip when the GPU path is asked for and unavailable;
    # this only guards the CPU-only suite from accidentally selecting them.
    pass


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import cpu

    cpu.build()
    return cpu
