import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine's kernels")


def _ensure_built():
    from cppqed_b200 import build
    if not os.path.exists(build.LIB):
        build.build()
    from tests import oracle_lib
    if not os.path.exists(oracle_lib.PATH):
        oracle_lib.build_oracle()


@pytest.fixture(scope="session")
def engine():
    _ensure_built()
    import cppqed_b200
    cppqed_b200.lib()
    return cppqed_b200


@pytest.fixture(scope="session")
def oracle():
    _ensure_built()
    from tests import oracle_lib
    return oracle_lib.Oracle()


@pytest.fixture(scope="session")
def golden():
    return json.load(open(os.path.join(ROOT, "tests", "golden", "reference_runs.json")))


@pytest.fixture(scope="session")
def gpu(engine):
    if engine.device_count() < 1:
        pytest.skip("no CUDA device")
    return engine
