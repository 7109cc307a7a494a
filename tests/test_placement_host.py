"""GpuBackend's placement wiring on the host, with a recording stand-in for
the engine library (no GPU): the automatic rule's modes reach dct_init3 for
v1-table cells and dct_b200_init3wm for wide-table cells, explicit modes
override the rule, and an all-HBM wide cell keeps plain dct_init3w."""
import pytest

import coldcore_b200.gpu as gpu


class Recorder:
    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        if not name.startswith("dct_"):
            raise AttributeError(name)

        def call(*args):
            self.calls.append((name, args))
            return 0
        return call


@pytest.fixture
def lib(monkeypatch):
    rec = Recorder()
    monkeypatch.setattr(gpu, "load_plugin", lambda path=None: rec)
    return rec


def _init_call(lib):
    return next(c for c in lib.calls if "init" in c[0])


def test_v1_cell_fits_hbm(lib):
    gpu.GpuBackend([3] * 8, 2)
    name, args = _init_call(lib)
    assert name == "dct_init3" and args[8:10] == (0, 0)


def test_v1_cell_over_budget_streams(lib, monkeypatch):
    # 6561 words: 91,854 B in all, 39,366 B for cnt and the map
    monkeypatch.setattr(gpu, "HBM_BUDGET", 50_000)
    b = gpu.GpuBackend([3] * 8, 2)
    name, args = _init_call(lib)
    assert name == "dct_init3" and args[8:10] == (1, 0)
    assert (b.layers_mode, b.cnt_mode) == (1, 0)
    lib.calls.clear()
    monkeypatch.setattr(gpu, "HBM_BUDGET", 30_000)
    gpu.GpuBackend([3] * 8, 2)
    assert _init_call(lib)[1][8:10] == (1, 1)


def test_explicit_modes_override(lib, monkeypatch):
    monkeypatch.setattr(gpu, "HBM_BUDGET", 10_000)
    gpu.GpuBackend([3] * 8, 2, layers_mode=0, cnt_mode=0)
    assert _init_call(lib)[1][8:10] == (0, 0)


def test_wide_cell_placement(lib, monkeypatch):
    gpu.GpuBackend([2] * 18, 2)                     # 18 axes: wide table
    assert _init_call(lib)[0] == "dct_init3w"
    lib.calls.clear()
    monkeypatch.setattr(gpu, "HBM_BUDGET", 2_000_000)   # 6|X| < 2 MB < 14|X|
    gpu.GpuBackend([2] * 18, 2)
    name, args = _init_call(lib)
    assert name == "dct_b200_init3wm" and args[-2:] == (1, 0)
