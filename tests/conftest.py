import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def pytest_collection_modifyitems(config, items):
    # GPU tests fail loudly when CUDA is missing instead of silently skipping,
    # unless they were deselected with -m "not gpu".
    pass


@pytest.fixture(scope="session")
def cuda_available():
    import torch
    return torch.cuda.is_available()
