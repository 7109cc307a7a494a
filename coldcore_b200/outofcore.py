"""Transforms of cells whose distance layers exceed device memory.

The reference places the layer planes of such a cell in host memory and
keeps cnt in HBM (``src/coldcore/gpu.py:253-260``); its kernels then read
the host planes over GH200's coherent C2C link
(``src/plugins/covering/dctcore_core.cuh:86-119``).  A B200 host link is not
coherent, so the engine streams the planes through device pieces with
explicit copies.  A transform is a product of per-axis recurrences, so the
axes can be applied in two phases, each of which touches the planes in
pieces that fit the device:

* phase 1, **slabs**: the low axes 0..s-1 act inside contiguous slabs of
  ``h`` whole rows of ``P_low = a_0 ... a_{s-1}`` words: a slab of every
  live plane is built on the device and copied out;
* phase 2, **columns**: the high axes s..n-1 act inside column blocks: the
  words ``[x0, x0 + w)`` of every one of the ``P_high = a_s ... a_{n-1}``
  rows, a pitched 2-D region (pitch ``P_low`` words) of each plane, copied
  in, transformed and written to the map or cnt in HBM.

Each live plane crosses the host link once per phase.  ``plan_pieces``
states the split rule that the engine's ``dct_b200_ooc_plan`` follows;
``ooc_plan``, ``ooc_record`` and ``ooc_transform`` call the engine (the
last one on a GPU).
"""
import ctypes
from math import prod

import numpy as np

MAX_PIECE_AXIS = 1 << 30          # a piece's own (slab-row / column) axis
MAX_PITCH = 2147483647            # bytes, the 2-D copy's row pitch
MIN_WIDTH = 32                    # columns of whole 128-byte rows at 4 B

PLAN_INFO = ("split", "p_low", "p_high", "slab_rows", "n_slabs", "col_width",
             "n_cols", "cap", "plane", "half", "live_mid", "host_bytes",
             "device_bytes", "link_bytes", "ball", "R1", "host_word_bytes")
REC_FIELDS = 20
OP_COPY, OP_COPY2D, OP_ZERO, OP_SCATTER, OP_LAUNCH, OP_JOIN = range(1, 7)
BUF_HOST, BUF_PIECE0, BUF_PIECE1, BUF_STAGE0, BUF_STAGE1, BUF_CODE, \
    BUF_CNT, BUF_OUT = range(8)


def plan_pieces(axes, cap, min_width=MIN_WIDTH, max_pitch_words=None):
    """The split and the piece sizes for pieces of at most ``cap`` words a
    plane: the largest low block ``P_low`` whose one-row slab fits (and
    whose row pitch a 2-D copy accepts) such that a column block of
    ``min(min_width, P_low)`` words of every high row fits too; then the
    most rows a slab and the widest column (whole multiples of
    ``min_width``) that fit.  Raises ``ValueError`` when no split fits."""
    axes = [int(a) for a in axes]
    if not axes or min(axes) < 1:
        raise ValueError("axes must be positive")
    if max_pitch_words is None:
        max_pitch_words = MAX_PITCH // 4
    size = prod(axes)
    best = None
    p_low = 1
    for s in range(1, len(axes)):
        p_low *= axes[s - 1]
        if p_low > cap or p_low > max_pitch_words:
            break
        p_high = size // p_low
        if cap // p_high >= min(min_width, p_low):
            best = (s, p_low, p_high, cap // p_high)
    if best is None:
        raise ValueError(f"no two-phase split of {axes} fits pieces of "
                         f"{cap} words")
    s, p_low, p_high, width_cap = best
    h = max(1, min(p_high, cap // p_low, MAX_PIECE_AXIS))
    w = min(p_low, width_cap, MAX_PIECE_AXIS)
    if w >= min_width:
        w -= w % min_width
    return {"split": s, "p_low": p_low, "p_high": p_high,
            "slab_rows": h, "n_slabs": -(-p_high // h),
            "col_width": w, "n_cols": -(-p_low // w)}


def plan_stream(axes, nlayers, bytes_per_word, budget_bytes, buffers=2,
                min_width=MIN_WIDTH):
    """``plan_pieces`` for a device budget in bytes: ``buffers`` pieces of
    ``nlayers`` planes of ``bytes_per_word`` resident at once.  Adds
    ``host_words``, the words both phases move over the host link."""
    if nlayers < 1 or bytes_per_word < 1 or buffers < 1:
        raise ValueError("nlayers, bytes_per_word and buffers must be >= 1")
    cap = int(budget_bytes) // (int(nlayers) * int(bytes_per_word)
                                * int(buffers))
    if cap < 1:
        raise ValueError("budget below one word of every layer")
    plan = plan_pieces(axes, cap, min_width)
    plan["host_words"] = 4 * nlayers * prod(int(a) for a in axes)
    return plan


def slabs(plan):
    """Phase-1 pieces: (first word, words) of each contiguous slab."""
    step = plan["slab_rows"] * plan["p_low"]
    total = plan["p_low"] * plan["p_high"]
    return [(x, min(step, total - x)) for x in range(0, total, step)]


def columns(plan):
    """Phase-2 pieces: (first low word, width) of each column block; the
    block is that range of every one of the ``p_high`` rows."""
    w, p_low = plan["col_width"], plan["p_low"]
    return [(x, min(w, p_low - x)) for x in range(0, p_low, w)]


# ------------------------------------------------------------ engine calls
def _lib(plugin_path=None):
    from .gpu import load_plugin
    lib = load_plugin(plugin_path)
    if not hasattr(lib, "dct_b200_ooc_plan"):
        raise RuntimeError("engine library lacks the out-of-core entry points")
    return lib


def _cell_args(problem, axes, R):
    from .patterns import PROBLEM_IDS
    ax = (ctypes.c_int * len(axes))(*[int(a) for a in axes])
    return PROBLEM_IDS[problem], len(axes), ax, int(R)


def _code_array(code):
    if code is None:
        return np.zeros(0, dtype=np.int64)
    return np.ascontiguousarray(np.atleast_1d(code), dtype=np.int64)


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))


def ooc_plan(problem, axes, R, init_mode, out_mode, device_budget, M=0,
             maxmult=1, min_width=0, plugin_path=None):
    """The engine's piece plan and memory needs (``PLAN_INFO``), no GPU."""
    lib = _lib(plugin_path)
    info = np.zeros(len(PLAN_INFO), dtype=np.int64)
    rc = lib.dct_b200_ooc_plan(*_cell_args(problem, axes, R), int(init_mode),
                               int(out_mode), int(M), int(maxmult),
                               int(device_budget), int(min_width), _ptr(info),
                               len(info))
    if rc:
        raise RuntimeError(f"dct_b200_ooc_plan rc={rc}")
    return dict(zip(PLAN_INFO, (int(v) for v in info)))


def ooc_record(problem, axes, R, init_mode, out_mode, device_budget,
               code=None, mu=1, min_width=0, plugin_path=None):
    """The engine's schedule for one streamed transform, without a GPU:
    an (ops, ``REC_FIELDS``) int64 array in issue order."""
    lib = _lib(plugin_path)
    code = _code_array(code)
    args = (*_cell_args(problem, axes, R), int(init_mode), int(out_mode),
            int(mu), _ptr(code), len(code), int(device_budget),
            int(min_width))
    n = lib.dct_b200_ooc_record(*args, None, 0)
    if n < 0:
        raise RuntimeError(f"dct_b200_ooc_record rc={n}")
    rows = np.zeros((max(n, 1), REC_FIELDS), dtype=np.int64)
    m = lib.dct_b200_ooc_record(*args, _ptr(rows), n)
    if m != n:
        raise RuntimeError(f"dct_b200_ooc_record gave {m} rows, then {n}")
    return rows[:n]


def ooc_transform(problem, axes, R, init_mode, out_mode, device_budget,
                  code=None, cnt=None, mu=1, min_width=0, host=None,
                  plugin_path=None):
    """One streamed transform on the current CUDA device.

    ``code`` (init 0) is a host word list; ``cnt`` (init 1 gain, 2 loss) a
    device tensor of |X| 16-bit counters; ``host`` an optional pinned uint8
    tensor of at least the plan's ``host_bytes`` to reuse across calls
    (pinning hundreds of GB takes seconds).  Returns ``(result, ms)``: the
    int32 map (out 1) or the cnt as int16 storage of uint16 values (out 2)
    as device tensors, or the (R+1, |X|) int32 layers in pinned host memory
    (out 3); ms the device time of the two phases."""
    import torch
    lib = _lib(plugin_path)
    code = _code_array(code)
    X = prod(int(a) for a in axes)
    mult = np.unique(code, return_counts=True)[1] if code.size else [0]
    plan = ooc_plan(problem, axes, R, init_mode, out_mode, device_budget,
                    M=len(code), maxmult=int(max(mult)),
                    min_width=min_width, plugin_path=plugin_path)
    if host is None:
        host = torch.empty(plan["host_bytes"], dtype=torch.uint8,
                           pin_memory=True)
    elif (host.dtype != torch.uint8 or host.is_cuda or
          not host.is_contiguous() or host.numel() < plan["host_bytes"]):
        raise ValueError("host must be a contiguous CPU uint8 tensor of at "
                         f"least {plan['host_bytes']} bytes")
    dev = torch.device("cuda", torch.cuda.current_device())
    out = None
    if out_mode == 1:
        out = torch.empty(X, dtype=torch.int32, device=dev)
    elif out_mode == 2:
        out = torch.empty(X, dtype=torch.int16, device=dev)
    cnt_ptr = None
    if init_mode != 0:
        if cnt is None or cnt.numel() != X or cnt.element_size() != 2 or \
                not cnt.is_cuda or not cnt.is_contiguous():
            raise ValueError("cnt must be a contiguous CUDA tensor of |X| "
                             "16-bit counters")
        cnt_ptr = cnt.data_ptr()
    ms = (ctypes.c_float * 2)()
    rc = lib.dct_b200_ooc_transform(
        *_cell_args(problem, axes, R), int(init_mode), int(out_mode), int(mu),
        _ptr(code), len(code), cnt_ptr,
        None if out is None else out.data_ptr(), host.data_ptr(),
        host.numel(), int(device_budget), int(min_width), ms)
    if rc:
        raise RuntimeError(f"dct_b200_ooc_transform rc={rc}")
    if out_mode == 3:
        layers = host.view(torch.int32)[:plan["R1"] * X].view(plan["R1"], X)
        return layers, (ms[0], ms[1])
    return out, (ms[0], ms[1])


def main(argv=None):
    """Time streamed coverage transforms (init 0, out 2) of one cell:
    ``python -m coldcore_b200.outofcore --axes 2x30 --R 3 --budget-gb 8``.
    Prints one JSON line: the plan, each rep's two phase times, and the
    host-link bytes per second of the fastest rep."""
    import argparse
    import json
    p = argparse.ArgumentParser(description=main.__doc__)
    p.add_argument("--problem", default="hamming")
    p.add_argument("--axes", default="2x30",
                   help="QxN for N axes of size Q, or a comma list")
    p.add_argument("--R", type=int, default=3)
    p.add_argument("--budget-gb", type=float, default=8.0)
    p.add_argument("--code", type=int, default=100000,
                   help="random code words (distinct)")
    p.add_argument("--reps", type=int, default=3)
    a = p.parse_args(argv)
    if "x" in a.axes:
        q, n = (int(v) for v in a.axes.split("x"))
        axes = [q] * n
    else:
        axes = [int(v) for v in a.axes.split(",")]
    X = prod(axes)
    rng = np.random.default_rng(1)
    code = np.unique(rng.integers(0, X, a.code))
    budget = int(a.budget_gb * 2 ** 30)
    plan = ooc_plan(a.problem, axes, a.R, 0, 2, budget, M=len(code),
                    maxmult=1)
    import torch
    host = torch.empty(plan["host_bytes"], dtype=torch.uint8, pin_memory=True)
    times = []
    for _ in range(a.reps):
        _, ms = ooc_transform(a.problem, axes, a.R, 0, 2, budget, code=code,
                              host=host)
        times.append([round(ms[0], 3), round(ms[1], 3)])
    best = min(t[0] + t[1] for t in times)
    print(json.dumps({"problem": a.problem, "axes": axes, "R": a.R,
                      "words": X, "plan": plan, "phase_ms": times,
                      "link_GBps": plan["link_bytes"] / best / 1e6,
                      "words_per_s": X / best * 1e3}))


if __name__ == "__main__":
    main()
