import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def native_lib():
    """The sm_100a library, built in-tree if it is missing (nvcc cross-compiles)."""
    from preprocess_src_b200 import _native
    if not _native.LIB_PATH.exists():
        from preprocess_src_b200 import build
        build.build()
    return _native.lib()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle
