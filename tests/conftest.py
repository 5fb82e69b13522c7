import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device of compute capability 10.x (B200)")
    config.addinivalue_line("markers", "slow: longer CPU-side checks")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def cuda_ctx():
    """A context on cuda:0.  GPU tests fail (not skip) when the library or the
    device is missing: the CUDA path is the product."""
    from spatialrust_b200 import _native
    from spatialrust_b200.csrc import build as csrc_build
    csrc_build.build()
    ctx = _native.shared_context(0)
    yield ctx
