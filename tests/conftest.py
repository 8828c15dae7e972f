import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "lb-cube_b200"), os.path.join(ROOT, "oracle"), os.path.dirname(__file__)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def engine():
    """The engine binding with its library built; the GPU tests use it."""
    import lbcube

    if not os.path.exists(lbcube.LIB_PATH):
        import build

        build.build()
    lbcube.load()
    return lbcube


@pytest.fixture(scope="session")
def dev():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without a CUDA device")
    return torch.device("cuda:0")
