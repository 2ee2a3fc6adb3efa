import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "p-milos_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the CUDA library and the oracle if they are missing (nvcc/gcc only)."""
    from pmilos_b200 import _build
    import pyoracle

    _build.build()
    pyoracle.build()
    yield


@pytest.fixture(scope="session")
def has_gpu():
    import torch

    return torch.cuda.is_available()
