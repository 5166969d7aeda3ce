import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long CPU run (full golden curves)")


def pytest_collection_modifyitems(config, items):
    if "slow" in (config.getoption("-m") or ""):
        return
    skip_slow = pytest.mark.skip(reason="slow: select with -m slow")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip_slow)


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def cuda_lib():
    """The in-tree CUDA library, built if needed; GPU tests fail (not skip)
    when it cannot be loaded, so a missing extension is never silent."""
    from plasticity_b200 import build as B
    from plasticity_b200 import capi
    B.build()
    return capi.load_library()
