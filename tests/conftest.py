import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def solver():
    """One CUDA context for the GPU tests (fails loudly when the library or device is missing)."""
    from tomostar_b200.eikonal import EikonalCuda

    s = EikonalCuda.create(0, 64)
    yield s
    s.close()
