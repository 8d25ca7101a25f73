import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the library's kernels")
    config.addinivalue_line("markers", "slow: longer CPU or GPU run")


def pytest_collection_modifyitems(config, items):
    # Tests that need no GPU must not be skipped silently when one is missing;
    # GPU tests are selected with -m gpu.
    pass


@pytest.fixture(scope="session")
def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
