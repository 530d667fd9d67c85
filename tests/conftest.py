import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) GPU")


def _built():
    from tagmatch_b200 import build
    return all(os.path.exists(p) for p in (build.LIB, build.WORKLOAD_LIB, build.FACADE_TEST, build.SERVE_BENCH, build.DRIVER))


@pytest.fixture(scope="session", autouse=True)
def native_libs():
    """Builds the in-tree libraries when they are missing (nvcc cross-compiles without a GPU)."""
    from tagmatch_b200 import build
    if not _built():
        build.build_all(quick=True)
    oracle_lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(oracle_lib):
        build.build_oracle()
    yield


def golden(name):
    return os.path.join(GOLDEN, name)
