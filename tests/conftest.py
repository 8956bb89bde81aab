import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build libculipx (sm_100a, cross-compiled) and the CPU oracle once per session."""
    from culip_b200 import build as cb_build
    from oracle import build as orc_build

    cb_build.build()
    orc_build.build()
    yield
