import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build libpfxtrace.so (sm_100a) and the CPU oracle once per session."""
    from pfx_b200 import build as product_build
    import oracle
    product_build.build()
    oracle.build()
    yield


def has_gpu() -> bool:
    from pfx_b200 import abi
    return abi.load().pfxt_device_count() > 0


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.fail("this test needs a CUDA device; run it with -m gpu on a GPU host")
    return True
