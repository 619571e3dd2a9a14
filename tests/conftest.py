import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA engine)")
    config.addinivalue_line("markers", "slow: full-size workloads")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build()
    return oracle


@pytest.fixture(scope="session")
def engine():
    """The CUDA engine through its C ABI; fails loudly if the library or the GPU is missing."""
    from partc_b200 import _lib
    from partc_b200 import build as b
    if not os.path.exists(_lib.LIB_PATH):
        b.build()
    assert _lib.device_count() > 0, "no sm_100 device visible to the engine"
    return _lib
