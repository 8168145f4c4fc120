"""Shared pytest configuration.

``@pytest.mark.gpu`` tests need a CUDA device. They are skipped only when the machine has
no CUDA device at all (probed through the driver library, without the engine), so on a GPU
machine a missing or broken native engine makes them fail instead of silently skipping.
"""
import ctypes
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _cuda_device_present() -> bool:
    try:
        cuda = ctypes.CDLL("libcuda.so.1")
    except OSError:
        return False
    if cuda.cuInit(0) != 0:
        return False
    n = ctypes.c_int(0)
    return cuda.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0


HAS_GPU = _cuda_device_present()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built native engine")
    config.addinivalue_line("markers", "slow: long-running")


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device on this machine")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
