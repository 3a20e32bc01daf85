import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running check")


def _cuda_device_count() -> int:
    try:
        import ctypes
        rt = ctypes.CDLL("libcuda.so.1")
        if rt.cuInit(0) != 0:
            return 0
        n = ctypes.c_int(0)
        if rt.cuDeviceGetCount(ctypes.byref(n)) != 0:
            return 0
        return n.value
    except OSError:
        return 0


HAS_GPU = _cuda_device_count() > 0


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device visible")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _native_libraries():
    """Build the in-tree native libraries once per session if they are missing or stale."""
    from helix_b200 import build as hb
    from oracle import build as ob
    hb.build()
    ob.build_oracle()
    ob.build_ref_host()
    ob.build_ref_cuda()
    yield


@pytest.fixture(scope="session")
def golden():
    import json

    def load(name):
        with open(os.path.join(GOLDEN, name)) as f:
            return json.load(f)
    return load
