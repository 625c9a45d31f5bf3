import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__ as entry  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the C-ABI kernels")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def fdr():
    return entry.load_package()


@pytest.fixture(scope="session")
def oracle():
    return entry.load_oracle()


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "runtests_known_answers.json")) as fh:
        return json.load(fh)


@pytest.fixture(autouse=True)
def _no_debug_index_violation(request):
    """Under the debug build (FDR_B200_DEBUG=1) every GPU test must end without a recorded
    index-check violation."""
    yield
    if os.environ.get("FDR_B200_DEBUG") != "1" or "gpu" not in request.keywords or not _has_gpu():
        return
    import ctypes as C
    lib = entry.load_package()._lib.lib()
    assert lib.fdr_debug_build() == 1
    w = C.c_uint64()
    assert lib.fdr_debug_fault(C.byref(w), None) == 0
    assert w.value == 0, f"index check failed: unit {(w.value >> 32) & 0x7fffffff}, line {w.value & 0xffffffff}"
