import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(__file__))
from _load import load_oracle, load_pkg  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu on a B200)")


@pytest.fixture(scope="session")
def dem():
    return load_pkg()


@pytest.fixture(scope="session")
def orc():
    return load_oracle()


@pytest.fixture(scope="session")
def wl(dem):
    import dem_b200.workloads as w
    return w


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test needs CUDA")
    torch.cuda.init()
    return torch
