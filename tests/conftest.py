import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


@pytest.fixture(scope="session")
def cuda_lib():
    """The in-tree CUDA library, built if missing. GPU tests fail (not skip)
    when no device is visible: there is no CPU fallback to test instead."""
    from ramses_b200 import build, runtime
    if not runtime.LIB_PATH.exists():
        build.build()
    L = runtime.load()
    assert L.rb_device_count() > 0, "no CUDA device visible to the CUDA library"
    return L


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle.lib()
