"""Per-operation timing: incremental updates, per-candidate gathers and the
fields of the non-Hamming cells.

Cells and operations (seeded, ``coldcore_b200.workloads``):

* binary Hamming n=26 R=3 and ternary n=16 R=4 at ~60% coverage: 1,000
  single-word add/remove updates, one ABI call per word, as the search core
  issues them;
* Lee Z_7^8 R=4 and the king 2048x2048 torus R=1 at 3% density: the
  recount / gain / loss fields (per launch, with the algorithmic bytes of
  each launch), 10^5 uniformly random candidates through ``ball_gather``
  roles 0 and 1 in one call each, and 1,000 single-word updates;
* K_8(9,4) with 940 codewords, the cell of coldcore's published
  single-word update and gather x64 / x1024 latencies
  (``docs/benchmarks.md:36-39``): the same three operations.

Wherever the reference's own ABI-v1 plugin (built from its source for
sm_100a into ``oracle/_ref``) accepts the cell, it runs the same calls on
the same GPU, and the final cnt of both after the update sequence is
compared by checksum.  Times are wall-clock around the calls with the
device drained before and after (a gather returns its counts to the host,
so it is synchronous; an update of one word is not, and the drain at the
end charges its device work).  The CPU baseline runs the oracle's
ball walks (numpy, one thread) on a bounded sample of the same calls,
from the cnt that the C restatement's recount computes.

    python -m harness.ops_bench [--cells LEE_7_8_4,KING_2048] [--json out]
"""
import argparse
import hashlib
import json
import os
import statistics
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_covering.so")

#: coldcore's GH200 numbers for K_8(9,4), docs/benchmarks.md:36-39
PUBLISHED_K8_9_4 = {"update_us": 27.0, "gather64_ms": 0.23,
                    "gather1024_ms": 4.1, "hardware": "GH200 (H100-class)"}

UPDATE_CELLS = ("H2_26_3", "H3_16_4", "K8_9_4", "LEE_7_8_4", "KING_2048")
FIELD_CELLS = ("LEE_7_8_4", "KING_2048")
GATHER_CELLS = ("LEE_7_8_4", "KING_2048", "K8_9_4", "H3_16_4")
N_UPDATES = 1000
N_CANDS = 100_000


def _sync():
    import torch
    torch.cuda.synchronize()


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def time_updates(b, words, signs):
    """Mean wall microseconds of one single-word update call."""
    _sync()
    t0 = time.perf_counter()
    for w, s in zip(words.tolist(), signs.tolist()):
        b.ball_update(np.array([w], dtype=np.int64), s)
    _sync()
    return 1e6 * (time.perf_counter() - t0) / len(words)


def time_gather(b, cands, role, reps=3):
    """Median wall milliseconds of one ball_gather call over ``cands``."""
    b.ball_gather(cands[:64], role)                     # warm
    ts = []
    for _ in range(reps):
        _sync()
        t0 = time.perf_counter()
        b.ball_gather(cands, role)
        ts.append(1e3 * (time.perf_counter() - t0))
    return statistics.median(ts)


def time_fields(b, reps=20):
    """Per transform: median device ms (CUDA events on the engine's stream)
    and every launch's algorithmic bytes and mean device ms."""
    import torch
    stream = torch.cuda.ExternalStream(b.stream)
    lib = b._lib
    out = {}
    for name, (i, o) in (("recount", (0, 2)), ("gain", (1, 1)),
                         ("loss", (2, 1))):
        for _ in range(3):
            lib.dct_transform(i, o)
        ts = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if lib.dct_transform(i, o):
                raise RuntimeError("transform failed")
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        b.set_timing(True)
        per = []
        for _ in range(reps):
            lib.dct_transform(i, o)
            per.append(b.last_timings())
        b.set_timing(False)
        plan = b.plan(i, o)
        launches = []
        for k, row in enumerate(plan):
            ms = statistics.mean(p[k] for p in per if k < len(p))
            j0, nax, by, kid = (int(v) for v in row)
            launches.append({"axes": f"{j0}..{j0 + nax - 1}", "bytes": by,
                             "ms": round(ms, 5),
                             "GBps": round(by / (ms * 1e-3) / 1e9, 1),
                             "kernel": "window" if kid == -2 else kid})
        out[name] = {"ms": round(statistics.median(ts), 5),
                     "launches": launches}
    return out


def cpu_ops(cell, code, words, signs, cands, n_upd=100, n_cand=2000):
    """The oracle's numpy ball walks (one thread) on a bounded sample:
    ``n_upd`` updates and ``n_cand`` candidates per role, from the cnt of
    the C restatement's recount."""
    from oracle.cport import CPortCell
    from oracle.dp_oracle import OracleBackend
    c = CPortCell(list(cell.axes), cell.R, cell.problem)
    c.recount(code)
    o = OracleBackend(list(cell.axes), cell.R, problem=cell.problem,
                      dtype=np.int32)
    o._A = None                              # the walks need cnt only
    o.cnt = c.cnt.astype(np.int32)
    t0 = time.perf_counter()
    for w, s in zip(words[:n_upd].tolist(), signs[:n_upd].tolist()):
        o.ball_update([w], s)
    upd = 1e6 * (time.perf_counter() - t0) / n_upd
    res = {"update_us": round(upd, 1)}
    for role in (0, 1):
        t0 = time.perf_counter()
        o.ball_gather(cands[:n_cand], role)
        res[f"gather_role{role}_us_per_cand"] = round(
            1e6 * (time.perf_counter() - t0) / n_cand, 2)
    res.update({"cores": 1, "kind": "port",
                "sample": f"{n_upd} single-word updates and {n_cand} "
                          "candidates per role, numpy restatement of the "
                          "reference's CPU ball walks, one thread"})
    return res


def measure_cell(name, cpu=True):
    from coldcore_b200.gpu import GpuBackend
    from coldcore_b200.workloads import (CELLS, candidates, code_for,
                                         update_sequence)
    cell = CELLS[name]
    code = code_for(cell)
    words, signs = update_sequence(cell.size, code, N_UPDATES, 1000 + cell.seed)
    cands = candidates(cell.size, N_CANDS, 2000 + cell.seed)
    res = {"axes": f"{cell.axes[0]}^{len(cell.axes)}", "R": cell.R,
           "M": cell.M, "problem": cell.problem}

    def run(b, tag):
        r = {}
        b.recount(code)
        r["ball"] = int(b.ball_len)
        if name in FIELD_CELLS and tag == "engine":
            r["fields"] = time_fields(b)
            b.recount(code)
        if name in GATHER_CELLS:
            if name == "K8_9_4":
                r["gather64_ms"] = round(time_gather(b, cands[:64], 0), 4)
                r["gather1024_ms"] = round(time_gather(b, cands[:1024], 0), 4)
            else:
                for role in (0, 1):
                    ms = time_gather(b, cands, role)
                    r[f"gather_role{role}_ms"] = round(ms, 3)
                    r[f"gather_role{role}_us_per_cand"] = round(
                        1e3 * ms / len(cands), 4)
                    r[f"role{role}_ball_words_per_s"] = round(
                        len(cands) * b.ball_len / (ms * 1e-3), 1)
        if name in UPDATE_CELLS:
            r["update_us"] = round(time_updates(b, words, signs), 2)
            r["cnt_sha16_after_updates"] = _digest(b.read_cnt())
        return r

    with GpuBackend(list(cell.axes), cell.R, problem=cell.problem) as b:
        res.update(run(b, "engine"))
    if os.path.exists(REF_LIB) and max(cell.axes) <= 16 and \
            len(cell.axes) <= 16 and cell.M <= 65535:
        with GpuBackend(list(cell.axes), cell.R, problem=cell.problem,
                        plugin_path=REF_LIB) as b:
            ref = run(b, "reference")
        ref["library"] = "oracle/_ref/libref_covering.so (reference " \
                         "dct_hc.cu, nvcc -O3 sm_100a)"
        res["reference_plugin"] = ref
        res["cnt_after_updates_equal"] = (
            ref.get("cnt_sha16_after_updates")
            == res.get("cnt_sha16_after_updates"))
    if name == "K8_9_4":
        res["published"] = PUBLISHED_K8_9_4
    if cpu and name in FIELD_CELLS:
        res["cpu_baseline"] = cpu_ops(cell, code, words, signs, cands)
    return res


def measure(cells=None, cpu=True):
    out = {}
    for name in cells or (UPDATE_CELLS + tuple(
            c for c in FIELD_CELLS if c not in UPDATE_CELLS)):
        try:
            out[name] = measure_cell(name, cpu=cpu)
        except Exception as e:                 # noqa: BLE001
            out[name] = {"error": f"{type(e).__name__}: {e}"}
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--cells", default=None)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--json", default=None)
    a = ap.parse_args()
    cells = a.cells.split(",") if a.cells else None
    res = measure(cells, cpu=not a.no_cpu)
    txt = json.dumps(res, indent=1)
    print(txt)
    if a.json:
        with open(a.json, "w") as f:
            f.write(txt)


if __name__ == "__main__":
    main()
