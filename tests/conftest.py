import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))
    return load


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device for gpu-marked tests; the native library must load."""
    import torch
    from tenex_b200 import native
    if not torch.cuda.is_available():
        pytest.fail("gpu test run without a CUDA device")
    native.lib()
    return torch.device("cuda:0")
