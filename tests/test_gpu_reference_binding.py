"""coldcore's own Python binding, search core and GPU test files driving
this engine's library unchanged.

The reference package and its test files sit in ``baseline/_ref`` (made by
``oracle/install_ref.py``, git-ignored, travelling with the working tree);
without them the module is skipped.  Every check compares the engine,
reached through the reference's ``coldcore.gpu.GpuBackend`` with
``plugin_path`` set to ``coldcore_b200/libcoldcore_covering.so``, against
the reference's own numpy backend (``coldcore.dp.NumpyDPBackend``):

* a K_3(8,2) session (fields, 100 updates, gathers of every role, the
  extraction and histogram queries) and Lee / torus / mu = 2 sessions;
* the optional and legacy symbols the binding feature-tests or may bind:
  ``dct_set_tbl2`` / ``dct_use_fmt`` (the ox support table, built by the
  reference's ``support_patterns_ox``), ``dct_init2`` / ``dct_init`` and
  ``dct_map_extract64``;
* the reference's ``Searcher`` (greedy, peel, LNS and the shell polish,
  whose moves are costed by the engine's ``swap_eval``), every state
  re-verified by the numpy backend;
* the reference's own GPU test files (``test_gpu_fast_paths``,
  ``test_gpu_counter_limits``, ``test_gpu_parity{,_lee,_torus,_grid,
  _multi}``) run in a child process with ``COLDCORE_PLUGIN_PATH`` naming
  this engine.

The engine keeps one cell per process (the ABI is a singleton), so every
session is closed before the next opens.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "baseline", "_ref")
LIB = os.path.join(ROOT, "coldcore_b200", "libcoldcore_covering.so")

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "coldcore")),
                       reason="reference package not installed "
                              "(python oracle/install_ref.py)")]

REF_GPU_FILES = ("test_gpu_fast_paths.py", "test_gpu_counter_limits.py",
                 "test_gpu_parity.py", "test_gpu_parity_lee.py",
                 "test_gpu_parity_torus.py", "test_gpu_parity_grid.py",
                 "test_gpu_parity_multi.py")


@pytest.fixture(scope="module")
def ref():
    """The reference modules, imported from baseline/_ref."""
    if REF not in sys.path:
        sys.path.insert(0, REF)
    import coldcore.dp
    import coldcore.gpu
    import coldcore.patterns
    import coldcore.search
    return coldcore


def _code(size, m, seed):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(size, size=m, replace=False)).astype(np.int64)


def _same_state(g, c):
    assert np.array_equal(np.asarray(g.read_cnt(), dtype=np.int64),
                          np.asarray(c.read_cnt(), dtype=np.int64))
    assert g.uncovered() == c.uncovered()


def _same_map(g, c, size):
    allw = np.arange(size, dtype=np.int64)
    gm = np.asarray(g.map_read_at(allw), dtype=np.int64)
    cm = np.asarray(c.map_read_at(allw), dtype=np.int64)
    assert np.array_equal(gm, cm)
    assert g.map_max() == c.map_max()
    mx = max(1, c.map_max())
    assert np.array_equal(np.asarray(g.map_hist(64, mx)),
                          np.asarray(c.map_hist(64, mx)))
    thr = max(1, mx // 2)
    gi, gv, gf = g.map_extract(thr, cap=1 << 16)
    ci, cv, cf = c.map_extract(thr, cap=1 << 16)
    assert gf == cf
    assert sorted(zip(np.asarray(gi).tolist(), np.asarray(gv).tolist())) == \
        sorted(zip(np.asarray(ci).tolist(), np.asarray(cv).tolist()))


@pytest.mark.parametrize("problem,axes,R,mu,m", [
    ("hamming", [3] * 8, 2, 1, 30), ("hamming", [3] * 8, 2, 2, 60),
    ("lee", [7] * 4, 2, 1, 40), ("torus_linf", [9, 7, 8], 1, 1, 25),
    ("hamming", [2, 3, 4, 5], 2, 1, 12)])
def test_reference_binding_session(ref, problem, axes, R, mu, m):
    size = int(np.prod(axes))
    code = _code(size, m, 7)
    c = ref.dp.NumpyDPBackend(axes, R, problem=problem, mu=mu)
    g = ref.gpu.GpuBackend(axes, R, problem=problem, plugin_path=LIB, mu=mu)
    try:
        g.recount(code)
        c.recount(code)
        _same_state(g, c)
        for t in range(4):
            assert g.count_eq(t) == c.count_eq(t)
        g.gain_map()
        c.gain_map()
        _same_map(g, c, size)
        g.loss_map()
        c.loss_map()
        _same_map(g, c, size)
        rng = np.random.default_rng(3)
        live = set(code.tolist())
        for step in range(100):
            if rng.random() < 0.5 or len(live) < 2:
                w = int(rng.integers(size))
                while w in live:
                    w = int(rng.integers(size))
                live.add(w)
                s = +1
            else:
                w = int(rng.choice(sorted(live)))
                live.discard(w)
                s = -1
            g.ball_update(np.array([w], dtype=np.int64), s)
            c.ball_update(np.array([w], dtype=np.int64), s)
            if step % 10 == 9:
                _same_state(g, c)
        probe = rng.integers(0, size, 257).astype(np.int64)
        for t in (0, 1, 2):
            assert np.array_equal(np.asarray(g.ball_gather(probe, t)),
                                  np.asarray(c.ball_gather(probe, t)))
        w = np.array([next(iter(live))], dtype=np.int64)
        delta = ref.gpu.ball_update_delta_generic
        assert g.ball_update_delta(w, -1) == delta(c, w, -1)
        assert g.ball_update_delta(w, +1) == delta(c, w, +1)
        drops = np.array(sorted(live)[:5], dtype=np.int64)
        cands = rng.integers(0, size, 40).astype(np.int64)
        gl, gg = g.swap_eval(drops, cands)
        cl, cg = ref.gpu.swap_eval_generic(c, drops, cands)
        assert np.array_equal(np.asarray(gl), np.asarray(cl))
        assert np.array_equal(np.asarray(gg), np.asarray(cg))
        _same_state(g, c)
    finally:
        g.close()


def test_ox_table_and_extract64(ref):
    """The ox support table (mask + nibble offsets) must give the same walks
    as the v1 table; dct_map_extract64 the same entries as dct_map_extract."""
    axes, R = [3] * 7, 2
    size = 3 ** 7
    code = _code(size, 25, 9)
    c = ref.dp.NumpyDPBackend(axes, R)
    g = ref.gpu.GpuBackend(axes, R, plugin_path=LIB)
    try:
        masks, offs = ref.patterns.support_patterns_ox(axes, R, "hamming")
        masks = np.ascontiguousarray(masks, dtype=np.uint16)
        offs = np.ascontiguousarray(offs, dtype=np.uint64)
        lib = g._lib
        assert lib.dct_set_tbl2(
            masks.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)),
            offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
            ctypes.c_longlong(len(masks))) == 0
        assert lib.dct_use_fmt(ctypes.c_int(1)) == 0
        g.recount(code)
        c.recount(code)
        rng = np.random.default_rng(4)
        for w in rng.integers(0, size, 30).tolist():
            g.ball_update(np.array([w], dtype=np.int64), +1)
            c.ball_update(np.array([w], dtype=np.int64), +1)
        _same_state(g, c)
        probe = rng.integers(0, size, 100).astype(np.int64)
        for t in (0, 1):
            assert np.array_equal(np.asarray(g.ball_gather(probe, t)),
                                  np.asarray(c.ball_gather(probe, t)))
        assert lib.dct_use_fmt(ctypes.c_int(0)) == 0
        g.gain_map()
        cap = 1 << 14
        i32 = np.zeros(cap, dtype=np.uint32)
        i64 = np.zeros(cap, dtype=np.int64)
        v32 = np.zeros(cap, dtype=np.int32)
        v64 = np.zeros(cap, dtype=np.int32)
        lib.dct_map_extract.restype = ctypes.c_longlong
        lib.dct_map_extract64.restype = ctypes.c_longlong
        n32 = lib.dct_map_extract(
            ctypes.c_int32(1), i32.ctypes.data_as(ctypes.c_void_p),
            v32.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(cap))
        n64 = lib.dct_map_extract64(
            ctypes.c_int32(1), i64.ctypes.data_as(ctypes.c_void_p),
            v64.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(cap))
        assert n32 == n64 > 0
        assert sorted(zip(i32[:n32].astype(np.int64).tolist(),
                          v32[:n32].tolist())) == \
            sorted(zip(i64[:n64].tolist(), v64[:n64].tolist()))
    finally:
        g.close()


@pytest.mark.parametrize("init", ["dct_init2", "dct_init"])
def test_legacy_inits(ref, init):
    """The homogeneous-Hamming inits the binding falls back to."""
    q, n, R = 3, 6, 1
    pats = ref.gpu.locality_order(
        ref.patterns.support_patterns([q] * n, R, "hamming"), [q] * n)
    pats = np.ascontiguousarray(pats, dtype=np.uint64)
    lib = ref.gpu.load_plugin(LIB)
    by = ctypes.c_longlong(0)
    pp = pats.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
    if init == "dct_init2":
        rc = lib.dct_init2(q, n, R, pp, ctypes.c_longlong(len(pats)), 4096,
                           ctypes.byref(by), 0, 0, 0)
    else:
        rc = lib.dct_init(q, n, R, pp, ctypes.c_longlong(len(pats)), 4096,
                          ctypes.byref(by))
    assert rc == 0 and by.value > 0
    try:
        code = _code(q ** n, 20, 5)
        c = ref.dp.NumpyDPBackend([q] * n, R)
        c.recount(code)
        assert lib.dct_set_code(code.ctypes.data_as(
            ctypes.POINTER(ctypes.c_longlong)), len(code)) == 0
        assert lib.dct_transform(0, 2) == 0
        cnt = np.zeros(q ** n, dtype=np.uint16)
        assert lib.dct_read_cnt(ctypes.c_longlong(0),
                                ctypes.c_longlong(q ** n),
                                cnt.ctypes.data_as(
                                    ctypes.POINTER(ctypes.c_uint16))) == 0
        assert np.array_equal(cnt.astype(np.int64),
                              np.asarray(c.read_cnt(), dtype=np.int64))
    finally:
        lib.dct_free()


@pytest.mark.parametrize("problem,axes,R", [
    ("hamming", [3] * 8, 2), ("hamming", [2] * 12, 2), ("lee", [5] * 5, 2)])
def test_reference_searcher_on_the_engine(ref, problem, axes, R):
    """The reference's search core on the engine: a greedy cover, peel, an
    LNS pass one notch down and the shell polish (its moves costed by the
    engine's swap_eval); each final state is recounted by the numpy
    backend, and the greedy cover is within two words of the one the same
    seed builds on the numpy backend (extraction order may differ, as in
    the reference's own GPU parity test)."""
    size = int(np.prod(axes))
    sizes = {}
    for name in ("engine", "numpy"):
        b = (ref.gpu.GpuBackend(axes, R, problem=problem, plugin_path=LIB)
             if name == "engine"
             else ref.dp.NumpyDPBackend(axes, R, problem=problem))
        try:
            s = ref.search.Searcher(b, seed=42)
            s.build_reserve_s = s.loop_reserve_s = 0.0
            s.load(np.zeros(0, dtype=np.int64))
            assert s.greedy_fill(10 ** 6) == 0
            s.peel()
            assert s.verify_full() == 0
            sizes[name] = len(s.code)
            if name == "engine":
                M = len(s.code) - 1
                unc = s.lns(M, 5.0, log_every=0)
                chk = ref.dp.NumpyDPBackend(axes, R, problem=problem)
                chk.recount(s.code)
                assert chk.uncovered() == unc == s.verify_full()
                unc = s.anneal(M, 3.0, mode="lahc", neighbourhood="shell",
                               log_every=0)
                chk.recount(s.code)
                assert chk.uncovered() == unc == s.verify_full()
                assert len(s.code) <= M
        finally:
            if name == "engine":
                b.close()
    assert abs(sizes["engine"] - sizes["numpy"]) <= 2
    assert size > 0


def test_reference_gpu_test_files_pass_on_the_engine():
    """The reference's own GPU suite, unchanged, in a child process with
    COLDCORE_PLUGIN_PATH naming this engine."""
    env = dict(os.environ, COLDCORE_PLUGIN_PATH=LIB, PYTHONPATH=REF)
    files = [os.path.join("tests", f) for f in REF_GPU_FILES]
    r = subprocess.run(
        [sys.executable, "-m", "pytest", "-c", os.devnull, "--rootdir", REF,
         "-p", "no:cacheprovider", "-q", "-W",
         "ignore::pytest.PytestUnknownMarkWarning", *files],
        cwd=REF, env=env, capture_output=True, text=True, timeout=1200)
    tail = (r.stdout + r.stderr)[-4000:]
    assert r.returncode == 0, tail
    import re
    m = re.search(r"(\d+) passed", r.stdout)
    assert m and int(m.group(1)) >= 100, tail      # they ran, not skipped
