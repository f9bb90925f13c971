import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """The product library and the C restatement oracle, built in-tree."""
    from graphic_lab_task_b200.build import build
    build()
    import pyoracle
    if not os.path.exists(pyoracle.PORT_SO):
        pyoracle.build(with_reference=False)
    yield


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected but torch.cuda.is_available() is False")
    torch.cuda.init()
    return torch
