import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100a) device")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def ctx():
    from libvc1_b200.api import CudaComputeContext

    c, err = CudaComputeContext.create(0)
    if c is None:
        pytest.fail(f"CUDA backend unavailable on a GPU test run: {err}")
    yield c
    c.close()
