import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


@pytest.fixture(scope="session")
def built_lib():
    """The in-tree CUDA library, compiled here if missing (nvcc cross-compiles)."""
    from splatfield_b200 import build

    path = build.LIB
    if not os.path.exists(path):
        build.build()
    return path


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def ctx(built_lib):
    import splatfield_b200 as sf

    return sf.default_context()
