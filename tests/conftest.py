import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "p-milos_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    """Register the gpu marker; build the CUDA library and the oracle if they are
    missing or stale (nvcc/gcc only) before any test module loads them."""
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")
    from pmilos_b200 import _build
    import pyoracle

    _build.build()
    pyoracle.build()


@pytest.fixture(scope="session")
def has_gpu():
    import torch

    return torch.cuda.is_available()
