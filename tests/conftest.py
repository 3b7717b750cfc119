import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200 / sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built_oracle():
    """The CPU oracle is test infrastructure; build it once per session."""
    from oracle import oracle
    if not os.path.exists(oracle.LIB_PATH):
        oracle.build()
    yield


def has_gpu() -> bool:
    try:
        from everest_b200 import capi
        return capi.device_count() > 0
    except Exception:
        return False
