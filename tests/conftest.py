import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA engine)")


@pytest.fixture(scope="session")
def engine_lib():
    """The built engine library (built on demand; no GPU needed to load it)."""
    from echidna_b200 import build, _lib
    if not os.path.exists(_lib.LIB_PATH):
        build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def ctx(engine_lib):
    from echidna_b200.gpu import CudaContext
    c = CudaContext.new()
    if c is None:
        pytest.fail("no CUDA device: GPU tests must run on a B200")
    yield c
    c.close()
