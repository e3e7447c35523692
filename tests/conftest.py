import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "tests" / "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import cpu_engine

    cpu_engine.build()
    return cpu_engine


@pytest.fixture(scope="session")
def engine_lib():
    from rfnetwork_b200 import _lib, build

    build.build()
    return _lib.load()
