"""Test configuration: the `gpu` marker and in-tree build of the libraries."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200, sm_100a) device")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    from tlfea_b200 import build

    build.build_oracle()
    if not build.LIB.exists():
        build.build_library()
    yield
