"""The engine against the reference's own kernels on the same B200.

``oracle/build_ref.py`` compiles the reference's ABI-v1 plugin
(src/plugins/covering/dct_hc.cu) for sm_100a into ``oracle/_ref``.  Both
libraries are driven through the same binding, on the same seeded inputs,
over the cells the reference accepts (axes <= 16, n <= 16, <= 65,535
occurrences; torus n <= 8), and every field, gather, update and query must
agree bit for bit.  Skipped when the reference library was not built."""
import os

import numpy as np
import pytest

from coldcore_b200.gpu import GpuBackend

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(
    __file__))), "oracle", "_ref", "libref_covering.so")

CELLS = [("hamming", [3] * 8, 2, 1, 30), ("hamming", [2] * 12, 3, 1, 60),
         ("hamming", [4, 4, 5, 5, 3], 2, 2, 40), ("hamming", [3] * 14, 3, 1,
                                                   1300),
         ("lee", [5, 6, 7, 4], 2, 1, 25), ("lee", [7] * 5, 3, 1, 60),
         ("torus_linf", [7, 9, 11], 2, 1, 20), ("torus_linf", [5, 5, 5], 1, 2,
                                                  15)]


@pytest.fixture(scope="module")
def ref_path():
    if not os.path.exists(REF):
        pytest.skip("reference plugin not built (oracle/build_ref.py)")
    return REF


def _map(b, ref):
    if ref:
        return b.map_read_at(np.arange(b.space.size, dtype=np.int64))
    return b.map_all()


@pytest.mark.parametrize("cell", CELLS,
                         ids=lambda c: f"{c[0]}-{c[1]}-R{c[2]}-mu{c[3]}")
def test_engine_matches_reference_plugin(ref_path, cell):
    prob, axes, R, mu, M = cell
    size = int(np.prod(axes))
    rng = np.random.default_rng(size + R + 7 * mu)
    code = np.sort(rng.choice(size, size=M, replace=False))
    if mu > 1:
        code = np.sort(np.concatenate([code, code[: M // 3]]))
    cand = rng.integers(0, size, 4000)
    upd = rng.choice(np.unique(code), size=min(10, len(code)), replace=False)
    add = rng.integers(0, size, 10)
    res = {}
    for name, path in (("ref", ref_path), ("ours", None)):
        r = res[name] = {}
        with GpuBackend(axes, R, problem=prob, mu=mu, plugin_path=path) as b:
            b.recount(code)
            r["cnt"] = b.read_cnt().copy()
            r["unc"] = b.uncovered()
            r["eq1"] = b.count_eq(1)
            b.gain_map()
            r["gain"] = _map(b, name == "ref")
            r["gmax"] = b.map_max()
            r["hist"] = b.map_hist(64, max(1, r["gmax"]))
            b.loss_map()
            r["loss"] = _map(b, name == "ref")
            r["g0"] = b.ball_gather(cand, 0)
            r["g1"] = b.ball_gather(cand, 1)
            b.ball_update(upd, -1)
            b.ball_update(add, +1)
            r["cnt2"] = b.read_cnt().copy()
            r["g0b"] = b.ball_gather(cand, 0)
            drops = np.unique(np.setdiff1d(code, upd))[:4]
            r["swap"] = b.swap_eval(drops, cand[:50])
    a, o = res["ref"], res["ours"]
    for k in ("cnt", "gain", "loss", "g0", "g1", "cnt2", "g0b", "hist"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(o[k])), k
    for k in ("unc", "eq1", "gmax"):
        assert a[k] == o[k], k
    assert np.array_equal(a["swap"][0], o["swap"][0])
    assert np.array_equal(a["swap"][1], o["swap"][1])
