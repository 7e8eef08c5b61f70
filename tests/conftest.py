import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


@pytest.fixture(scope="session", autouse=True)
def _native_built():
    """Build (or verify) the in-tree native libraries once per session."""
    from empanada_b200 import build

    build.build_native()
    from oracle import bind

    if not os.path.exists(bind.LIB_PATH):
        bind.build()
    yield


@pytest.fixture(scope="session")
def engine():
    import empanada_b200

    eng = empanada_b200.Engine(0)
    yield eng
    eng.close()
