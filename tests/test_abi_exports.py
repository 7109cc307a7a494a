"""The engine library loads on a machine without a GPU and exports every
symbol the public header declares; entry points that need no device
answer their documented errors."""
import ctypes
import os
import re

import numpy as np

from coldcore_b200 import build
from coldcore_b200.gpu import REQUIRED, load_plugin

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "coldcore_b200", "plugin.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(dct_\w+)\s*\(", text)))


def test_library_builds_and_exports_every_declared_symbol():
    path = build.build()
    lib = ctypes.CDLL(path)
    names = declared()
    assert len(names) >= 31
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    for n in REQUIRED:
        assert n in names


def test_header_cites_the_reference_for_every_v1_symbol():
    text = open(HEADER).read()
    for n in REQUIRED + ("dct_init2", "dct_init", "dct_set_mu",
                         "dct_ball_gather_mu", "dct_swap_eval"):
        lines = text.splitlines()
        i = next(k for k, ln in enumerate(lines)
                 if re.search(r"\b" + n + r"\s*\(", ln))
        near = "\n".join(lines[max(0, i - 5):i + 1])
        assert "plugin.h:" in near and "dct_hc.cu" in near, n


def test_calls_before_init_are_rejected_without_a_device():
    lib = load_plugin()
    assert lib.dct_get_mu() == 1
    assert lib.dct_transform(1, 1) == -1
    w = np.zeros(1, dtype=np.int64)
    assert lib.dct_set_code(w.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                            1) == -1
    assert lib.dct_set_mu(0) == -1
    assert lib.dct_set_mu(70000) == -1
