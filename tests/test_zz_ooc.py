"""Out-of-core transforms on the GPU (dct_b200_ooc_transform): the layer
planes streamed through small device pieces in pinned host memory give,
bit for bit, the oracle's map, cnt and layers on small cells cut into many
slabs and ragged columns, and the in-memory engine's on H2(22,3)."""
import numpy as np
import pytest

from coldcore_b200.outofcore import ooc_plan, ooc_transform
from oracle.dp_oracle import OracleBackend

pytestmark = [pytest.mark.gpu, pytest.mark.late(3)]

torch = pytest.importorskip("torch")


def _budget(R1, cap, out_mode, M):
    per = 2 * (R1 * 4 + (2 if out_mode == 2 else 0))
    return (cap + 64) * per + 8 * M


def _cnt_tensor(cnt):
    return torch.from_numpy(np.asarray(cnt, np.uint16).view(np.int16)).cuda()


# (family, axes, R, piece words a plane): several slabs and ragged columns
CELLS = [("hamming", [3] * 7, 2, 400), ("hamming", [2] * 12, 3, 400),
         ("lee", [5, 6, 7, 4], 3, 400), ("torus_linf", [5, 7, 6, 5], 2, 400),
         ("grid_linf", [4, 6, 5, 3], 2, 100),
         ("hamming", [4, 4, 4, 4, 4], 2, 400)]
MODES = [(0, 1), (0, 2), (0, 3), (1, 1), (1, 3), (2, 1), (2, 3)]


@pytest.mark.parametrize("problem,axes,R,cap", CELLS,
                         ids=lambda v: str(v).replace(" ", ""))
def test_streamed_modes_match_the_oracle(problem, axes, R, cap):
    layered = problem in ("hamming", "lee")
    R1 = R + 1 if layered else 1
    o = OracleBackend(axes, R, problem)
    rng = np.random.default_rng(3)
    code = rng.choice(o.space.size, o.space.size // 30, replace=False)
    code = np.concatenate([code, code[:3]])
    o.recount(code)
    cnt = o.cnt.astype(np.uint16)
    for init_mode, out_mode in MODES:
        if out_mode == 3 and not layered:
            continue
        M = len(code) if init_mode == 0 else 0
        budget = _budget(R1, cap, out_mode, M)
        info = ooc_plan(problem, axes, R, init_mode, out_mode, budget, M=M,
                        maxmult=2, min_width=4)
        assert info["n_slabs"] * info["n_cols"] > 2
        got, ms = ooc_transform(problem, axes, R, init_mode, out_mode,
                                budget, code=code if init_mode == 0 else None,
                                cnt=_cnt_tensor(cnt), min_width=4)
        if init_mode == 0:
            o.recount(code)
            want = o.cnt
        elif init_mode == 1:
            o.gain_map()
            want = o.map
        else:
            o.loss_map()
            want = o.map
        if out_mode == 3:
            assert np.array_equal(got.numpy(), o.layers()), init_mode
        elif out_mode == 2:
            assert np.array_equal(got.cpu().numpy().view(np.uint16), want)
        else:
            assert np.array_equal(got.cpu().numpy(), want), init_mode


def test_h2_22_3_against_the_in_memory_engine():
    from coldcore_b200.gpu import GpuBackend
    axes, R = [2] * 22, 3
    rng = np.random.default_rng(5)
    code = rng.choice(1 << 22, 20000, replace=False)
    budget = _budget(4, 1 << 18, 1, len(code))
    info = ooc_plan("hamming", axes, R, 0, 1, budget, M=len(code),
                    maxmult=1)
    assert info["n_slabs"] == 16 and info["n_cols"] == 16
    with GpuBackend(axes, R, "hamming") as g:
        g.recount(code)
        want_cnt = g.read_cnt()
        g.gain_map()
        want_gain = g.map_all()
        g.loss_map()
        want_loss = g.map_all()
    got, ms = ooc_transform("hamming", axes, R, 0, 2,
                            _budget(4, 1 << 18, 2, len(code)), code=code)
    cnt = got.cpu().numpy().view(np.uint16)
    assert np.array_equal(cnt, want_cnt)
    assert ms[0] > 0 and ms[1] > 0
    for init_mode, want in ((1, want_gain), (2, want_loss)):
        got, _ = ooc_transform("hamming", axes, R, init_mode, 1,
                               _budget(4, 1 << 18, 1, 0),
                               cnt=_cnt_tensor(cnt))
        assert np.array_equal(got.cpu().numpy(), want), init_mode


def _session(axes, R, problem, layers_mode, code):
    """Every transform kind and the reads after them, on one engine cell."""
    from coldcore_b200.gpu import GpuBackend
    r = {}
    with GpuBackend(axes, R, problem, layers_mode=layers_mode) as g:
        g.recount(code)
        r["cnt"] = g.read_cnt().copy()
        r["unc"] = g.uncovered()
        g.gain_map()
        r["gain"] = g.map_all().copy()
        r["gain_max"] = g.map_max()
        g.loss_map()
        r["loss"] = g.map_all().copy()
        if problem in ("hamming", "lee"):
            g.layers_map(0)
            r["layers"] = np.stack([g.layer(d) for d in range(R + 1)])
            r["at"] = g.layers_at(code[:7])
        g.ball_update(code[:2], -1)
        g.gain_map()
        r["gain2"] = g.map_all().copy()
        r["ext"] = np.sort(g.map_extract(1)[0])
    return r


# (family, axes, R, device KB): every transform of the session in at least
# two pieces (14-36 slabs, 12-41 columns on the layered cells); H2(18,2)
# takes the wide support table (dct_b200_init3wm)
HOST_CELLS = [("hamming", [3] * 9, 2, 48), ("lee", [6] * 6, 3, 72),
              ("torus_linf", [7, 9, 11], 2, 8), ("grid_linf", [8, 8, 8], 2, 4),
              ("hamming", [2] * 18, 2, 1024)]


@pytest.mark.parametrize("problem,axes,R,kb", HOST_CELLS,
                         ids=lambda v: str(v).replace(" ", ""))
def test_host_placement_matches_hbm(problem, axes, R, kb, monkeypatch):
    """layers_mode 1 (host planes, streamed) through the ordinary ABI: the
    same counts, maps, layers and queries as the HBM cell, with a device
    budget small enough for many pieces."""
    rng = np.random.default_rng(11)
    X = int(np.prod(axes))
    code = rng.choice(X, X // 40, replace=False)
    want = _session(axes, R, problem, 0, code)
    monkeypatch.setenv("CC_OOC_BUDGET_KB", str(kb))
    got = _session(axes, R, problem, 1, code)
    for k in want:
        assert np.array_equal(np.asarray(got[k]), np.asarray(want[k])), k
