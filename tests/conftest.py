import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (runs the CUDA library)")


@pytest.fixture(scope="session")
def gpu_ctx_factory():
    """Creates library contexts on cuda:0; skips nothing -- a missing GPU is a failure."""
    from hprmat_b200 import Context
    made = []

    def make(**kw):
        c = Context(**kw)
        made.append(c)
        return c

    yield make
    for c in made:
        c.close()
