"""Loader for the committed golden fixtures (written by
tests/golden/make_golden.py from the reference's own CPU backends)."""
import json
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

TRANSFORM_CELLS = [
    ([2] * 9, 3, 1), ([2] * 10, 2, 1), ([3] * 7, 2, 1), ([3] * 2, 1, 1),
    ([4] * 5, 4, 1), ([5] * 5, 3, 1), ([4, 4, 5, 5, 3], 2, 1),
    ([6] * 4, 2, 1), ([7] * 4, 3, 1), ([8] * 4, 4, 1), ([9] * 4, 3, 1),
    ([10] * 4, 4, 1), ([3] * 4, 4, 1), ([7] * 3, 3, 1),
    ([2, 3, 4, 5, 6, 7], 3, 1), ([10, 9, 8, 7, 6], 5, 1), ([3] * 6, 2, 2),
    ([4] * 4, 1, 3),
]

FAMILY_CELLS = [
    ("hamming", [3] * 6, 1, 1), ("hamming", [4] * 5, 2, 1),
    ("hamming", [3, 4, 5, 6], 2, 1), ("hamming", [3] * 5, 1, 2),
    ("hamming", [2, 3, 4], 1, 1), ("hamming", [3, 4, 5], 1, 3),
    ("hamming", [2, 2, 2, 2], 1, 2), ("hamming", [3, 3, 3], 2, 3),
    ("hamming", [3, 3], 1, 1),
    ("lee", [5, 6, 7], 2, 1), ("lee", [4, 4, 4, 4], 3, 1),
    ("lee", [5, 5], 1, 1), ("lee", [4, 6], 2, 2), ("lee", [3, 4, 5], 1, 1),
    ("lee", [4, 4, 4], 3, 1), ("lee", [16, 3, 2], 2, 1),
    ("torus_linf", [7, 9, 11], 2, 1), ("torus_linf", [9, 9], 1, 1),
    ("torus_linf", [5, 7], 1, 1), ("torus_linf", [6, 6], 1, 3),
    ("torus_linf", [5, 5, 5], 1, 2), ("torus_linf", [16, 3, 5], 1, 1),
    ("grid_linf", [4, 5, 6], 3, 1), ("grid_linf", [8, 8], 1, 2),
    ("grid_linf", [5, 9], 1, 1), ("grid_linf", [4, 4], 2, 1),
    ("grid_linf", [6, 3, 3], 1, 2), ("grid_linf", [3, 3], 3, 1),
    ("grid_linf", [16, 4], 1, 1),
]

WIDE_CELLS = [
    ("torus_linf", [250, 240], 1, 1), ("torus_linf", [250, 240], 2, 1),
    ("grid_linf", [250, 240], 1, 1), ("torus_linf", [33, 40, 17], 1, 1),
]

_cache = {}


def small():
    if "small" not in _cache:
        _cache["small"] = dict(np.load(os.path.join(HERE, "small_fields.npz")))
    return _cache["small"]


def tables():
    if "tables" not in _cache:
        _cache["tables"] = dict(np.load(os.path.join(HERE,
                                                     "support_tables.npz")))
    return _cache["tables"]


def full():
    with open(os.path.join(HERE, "full_configs.json")) as f:
        return json.load(f)


def cell_id(problem, axes, R, mu):
    return f"{problem}-{'x'.join(map(str, axes))}-R{R}-mu{mu}"


def key(*parts):
    return "__".join(str(p) for p in parts)


def incidence_golden():
    """The reference's explicit-incidence backends on seeded cells
    (make_incidence_golden.py)."""
    if "incidence" not in _cache:
        _cache["incidence"] = dict(np.load(os.path.join(
            HERE, "incidence_golden.npz")))
    return _cache["incidence"]


def incidence_cells():
    """Cell keys of incidence_golden(): dense*, design*, weighted*."""
    keys = {k.split("/")[0] for k in incidence_golden()}
    return sorted(keys)
