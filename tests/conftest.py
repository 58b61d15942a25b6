import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100) device")


def _cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle, build
    build(reference=True)
    return Oracle()


@pytest.fixture(scope="session")
def reference(oracle):
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("the reference harness (oracle/_ref) is not built")
    r = Reference()
    r.set_threads(1)
    return r


@pytest.fixture(scope="session")
def engine():
    from insiliscope_b200.build import build_library
    build_library()
    from insiliscope_b200 import Engine
    e = Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(ROOT, "tests", "golden")
