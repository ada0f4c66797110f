import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the sm_100a kernels")


@pytest.fixture(scope="session")
def ls():
    import lightspeed_b200
    return lightspeed_b200


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
