import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "serial_small.npz"))


@pytest.fixture(scope="session")
def backend():
    """The B200 backend on cuda:0; raises (never skips) when the GPU path is unusable."""
    from qtctreconstruction_b200 import B200Backend
    be = B200Backend(0)
    yield be
    be.close()
