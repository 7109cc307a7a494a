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
    # tests of code that has not yet passed on a B200 run after the others
    # (stable, by rank), so that a run stopping at the first failure has
    # run everything proven first
    def rank(item):
        m = item.get_closest_marker("late")
        return m.args[0] if m and m.args else (1 if m else 0)
    items[:] = sorted(items, key=rank)
    if gpu_present():
        return
    skip = pytest.mark.skip(reason="no CUDA device on this machine")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
