"""Shared test setup: the `gpu` marker, repository paths and GPU detection.

GPU detection asks the CUDA driver directly (libcuda via ctypes), so CPU-only runs never
import a framework or touch a device.
"""
import ctypes
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_count() -> int:
    try:
        cu = ctypes.CDLL("libcuda.so.1")
    except OSError:
        return 0
    if cu.cuInit(0) != 0:
        return 0
    n = ctypes.c_int(0)
    if cu.cuDeviceGetCount(ctypes.byref(n)) != 0:
        return 0
    return n.value


HAVE_GPU = gpu_count() > 0


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
