import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the native CUDA path")


@pytest.fixture(scope="session", autouse=True)
def _built_oracle():
    """The oracle's C restatement is rebuilt here when missing (a few seconds with gcc)."""
    from oracle import native
    if not os.path.exists(os.path.join(native.HERE, "liboracle.so")):
        native.build(ref=False)
    yield


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch.device("cuda:0")
