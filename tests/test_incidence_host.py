"""The explicit-incidence engine's host side, without a GPU: the ABI-2
library loads and exports every symbol its header declares, answers the
no-cell errors, and rejects malformed cells before touching the device; the
Python mirror validates its arguments the way coldcore's binding does."""
import ctypes
import os
import re

import numpy as np
import pytest

from coldcore_b200 import build
from coldcore_b200.incidence import (GpuIncidenceBackend,
                                     GpuWeightedIncidenceBackend,
                                     IncidenceSpace, load_sparse_plugin)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "coldcore_b200", "sparse.h")

LL, I32P, I64P = ctypes.c_longlong, ctypes.POINTER(ctypes.c_int32), \
    ctypes.POINTER(ctypes.c_int64)


@pytest.fixture(scope="module")
def lib():
    build.build_sparse()
    return load_sparse_plugin()


def test_exports_every_declared_symbol(lib):
    names = sorted(set(re.findall(r"\b(sparse_\w+)\s*\(", open(HEADER).read())))
    assert len(names) >= 23
    raw = ctypes.CDLL(build.SPARSE_LIB)
    assert [n for n in names if not hasattr(raw, n)] == []


def test_header_cites_the_reference_for_every_abi2_symbol():
    lines = open(HEADER).read().splitlines()
    for i, ln in enumerate(lines):
        m = re.search(r"\b(sparse_\w+)\s*\(", ln)
        if m and not m.group(1).startswith("sparse_b200_"):
            near = "\n".join(lines[max(0, i - 6):i + 1])
            assert "sparse.cu:" in near, m.group(1)


def test_no_cell_answers(lib):
    assert lib.sparse_abi_version() == 2
    assert lib.sparse_inc_mode() == -1 and lib.sparse_is_csr() == 0
    assert lib.sparse_free() == 0
    assert lib.sparse_field(0) == -1
    assert lib.sparse_count_eq(0) == -1 and lib.sparse_count_deficit() == -1
    out = np.zeros(4, dtype=np.int32)
    assert lib.sparse_read_cnt(0, 1, out.ctypes.data_as(I32P)) == -1
    assert lib.sparse_set_mu(0) == -1
    assert lib.sparse_set_mu(3) == 0 and lib.sparse_get_mu() == 3
    assert lib.sparse_set_mu(1) == 0
    assert lib.sparse_b200_row_lanes() == -1


def _init(lib, inc, n_univ, mode=0, cap=16, n_cand=None, d=None):
    inc = np.ascontiguousarray(inc, dtype=np.int32)
    n_cand = inc.shape[0] if n_cand is None else n_cand
    d = inc.shape[1] if d is None else d
    return lib.sparse_init(n_cand, d, n_univ, inc.ctypes.data_as(I32P), mode,
                           cap, None, None)


def test_malformed_dense_cells_are_rejected_before_the_device(lib):
    inc = np.array([[0, 1], [2, 3]], dtype=np.int32)
    assert _init(lib, inc, 4, n_cand=0) == -2
    assert _init(lib, inc, 4, d=0) == -2
    assert _init(lib, inc, 0) == -2
    assert _init(lib, inc, 4, mode=2) == -2
    assert _init(lib, inc, 4, cap=0) == -2
    assert _init(lib, inc, 3) == -2                  # entry 3 outside [0, 3)
    assert _init(lib, np.array([[0, -1]]), 4) == -2
    assert lib.sparse_init(2, 2, 4, None, 0, 16, None, None) == -2
    assert lib.sparse_inc_mode() == -1               # nothing was created


def _init_csr(lib, indptr, indices, w, uw, n_univ, n_cand=None, nnz=None):
    indptr = np.ascontiguousarray(indptr, dtype=np.int64)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    w = np.ascontiguousarray(w, dtype=np.int32)
    uw = np.ascontiguousarray(uw, dtype=np.int32)
    n_cand = len(indptr) - 1 if n_cand is None else n_cand
    nnz = len(indices) if nnz is None else nnz
    return lib.sparse_init_csr(n_cand, n_univ, nnz,
                               indptr.ctypes.data_as(I64P),
                               indices.ctypes.data_as(I32P),
                               w.ctypes.data_as(I32P), uw.ctypes.data_as(I32P),
                               0, 16, None, None)


def test_malformed_csr_cells_are_rejected_before_the_device(lib):
    ip, ix, w, uw = [0, 2, 3], [0, 1, 2], [1, 2, 1], [1, 1, 1]
    assert _init_csr(lib, [1, 2, 3], ix, w, uw, 3) == -2    # indptr[0] != 0
    assert _init_csr(lib, [0, 2, 2], ix, w, uw, 3) == -2    # end != nnz
    assert _init_csr(lib, [0, 3, 2, 3], ix, w, uw, 3) == -2  # decreasing
    assert _init_csr(lib, ip, [0, 1, 3], w, uw, 3) == -2    # index outside
    assert _init_csr(lib, ip, ix, [1, 0, 1], uw, 3) == -2   # weight 0
    assert _init_csr(lib, ip, ix, w, [1, 0, 1], 3) == -2    # uw 0
    assert _init_csr(lib, ip, ix, w, uw, 3, nnz=-1) == -2
    assert lib.sparse_inc_mode() == -1


def test_python_mirror_validates_like_the_reference():
    with pytest.raises(ValueError):
        GpuIncidenceBackend(np.zeros(4, dtype=np.int32), 4)
    with pytest.raises(ValueError):
        GpuIncidenceBackend(np.array([[0, 4]]), 4)
    with pytest.raises(ValueError):
        GpuIncidenceBackend(np.array([[0, 1]]), 4, mu=0)
    with pytest.raises(ValueError):
        GpuIncidenceBackend(np.array([[0, 1]]), 4, inc_mode=2)
    with pytest.raises(ValueError):
        GpuWeightedIncidenceBackend([0, 2], [0, 1], [1, 0], 3)
    with pytest.raises(ValueError):
        GpuWeightedIncidenceBackend([0, 3], [0, 1], [1, 1], 3)
    with pytest.raises(ValueError):
        GpuWeightedIncidenceBackend([0, 2], [0, 1], [1, 1], 3, uw=[1, 1])
    s = IncidenceSpace(5)
    assert s.index_word([3, 4]).shape == (2, 1)
    assert s.word_index(s.index_word([3, 4])).tolist() == [3, 4]
    with pytest.raises(ValueError):
        IncidenceSpace(0)


def test_design_constructor_name_serves_the_gpu_form_only():
    from coldcore_b200.incidence import CoveringDesignBackend
    with pytest.raises(ValueError):
        CoveringDesignBackend(7, 3, 2, device="cpu")
    with pytest.raises(ValueError):
        CoveringDesignBackend(7, 3, 2, device="ref")
