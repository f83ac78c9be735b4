import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libhdd_b200.so")


# Run order: the CPU tests, then the GPU parity, edge-case and serving suites,
# then the other GPU tests, and the allocation-free entry point's test last, so
# that a run stopping at its first failure (-x) has already run the main suites.
_CORE_GPU = ("test_gpu_parity.py", "test_gpu_c2_parity.py", "test_gpu_edge_cases.py", "test_gpu_server.py")


def pytest_collection_modifyitems(session, config, items):
    def rank(item):
        name = os.path.basename(str(item.fspath))
        if name == "test_zz_no_alloc.py":
            return 3
        if name.startswith("test_cpu_"):
            return 0
        return 1 if name in _CORE_GPU else 2
    items.sort(key=rank)


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def hdd_lib():
    from hierarchicaldd_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from hierarchicaldd_b200 import build
        build.build()
    return _lib.load()
