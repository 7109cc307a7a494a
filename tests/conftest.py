import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def gpu_present():
    return (os.path.exists("/dev/nvidia0") or os.path.exists("/dev/nvidiactl")
            or bool(os.environ.get("COLDCORE_FORCE_GPU_TESTS")))


def pytest_collection_modifyitems(config, items):
    if gpu_present():
        return
    skip = pytest.mark.skip(reason="no CUDA device on this machine")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
