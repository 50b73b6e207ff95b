"""Shared test setup: markers, import paths, built artefacts."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def _have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _have_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_c():
    import oracle
    oracle.build()
    return oracle.oracle()


@pytest.fixture(scope="session")
def reference():
    import oracle
    r = oracle.reference()
    if r is None:
        pytest.skip("reference CPU code not built here (oracle/_ref)")
    return r


@pytest.fixture(scope="session")
def lib():
    from image360_b200 import build, load_library
    if not os.path.exists(build.LIB):
        build.build()
    return load_library()


@pytest.fixture(scope="session")
def backend(lib):
    from image360_b200 import B200ComputeBackend, ComputeResult
    b = B200ComputeBackend()
    rc = b.initialize()
    assert rc == ComputeResult.SUCCESS, b.get_last_error()
    return b
