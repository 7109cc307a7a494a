#!/usr/bin/env python3
"""Generate the golden fixtures from the reference's own CPU backends.

Run in a checkout that has the reference source, with
``COLDCORE_REF_SRC`` naming its ``src/`` directory:

    python tests/golden/make_golden.py            # small fixtures (~1 min)
    python tests/golden/make_golden.py --full     # + full-size checksums

Outputs (committed; nothing at test time reads the reference):

``small_fields.npz``   complete cnt / gain / loss fields, gathers, update
                       traces and map queries of the reference's
                       ``coldcore.dp.NumpyDPBackend`` on small cells of all
                       four problem families (mu = 1..3), each cross-checked
                       here against the reference's brute-force backends
                       where the space allows;
``support_tables.npz`` the reference's packed v1 support tables
                       (``coldcore.patterns.support_patterns``) and their
                       locality order (``coldcore.gpu.locality_order``);
``full_configs.json``  SHA-256 checksums of the fields of the full-size
                       cells (H2(26,3), H3(16,4), Lee Z_7^8, king 2048^2 and
                       K_3(14,3)) and of the field after 1,000 seeded
                       updates, from the same reference backend.
"""
import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF_SRC = os.environ.get("COLDCORE_REF_SRC")
if not REF_SRC or not os.path.isdir(os.path.join(REF_SRC, "coldcore")):
    sys.exit("set COLDCORE_REF_SRC to the reference checkout's src/ "
             "directory (the one holding the coldcore package)")
sys.path.insert(0, REF_SRC)

from coldcore.dp import NumpyDPBackend                      # noqa: E402
from coldcore.gpu import locality_order                      # noqa: E402
from coldcore.patterns import support_patterns               # noqa: E402
from coldcore.reference import (RefGridBackend, RefHammingBackend,  # noqa
                                RefLeeBackend, RefTorusBackend)

from coldcore_b200.workloads import (CELLS, candidates, code_for,  # noqa
                                     update_sequence)

REF = {"hamming": RefHammingBackend, "lee": RefLeeBackend,
       "torus_linf": RefTorusBackend, "grid_linf": RefGridBackend}

# the Hamming transform cells of the reference's GPU fast-path tests
TRANSFORM_CELLS = [
    ([2] * 9, 3, 1), ([2] * 10, 2, 1), ([3] * 7, 2, 1), ([3] * 2, 1, 1),
    ([4] * 5, 4, 1), ([5] * 5, 3, 1), ([4, 4, 5, 5, 3], 2, 1),
    ([6] * 4, 2, 1), ([7] * 4, 3, 1), ([8] * 4, 4, 1), ([9] * 4, 3, 1),
    ([10] * 4, 4, 1), ([3] * 4, 4, 1), ([7] * 3, 3, 1),
    ([2, 3, 4, 5, 6, 7], 3, 1), ([10, 9, 8, 7, 6], 5, 1), ([3] * 6, 2, 2),
    ([4] * 4, 1, 3),
]

# every family, mixed radix, even/odd axes, oversized grid windows, mu > 1
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

# wide axes (above the reference plugin's 16-wide packed tables; below the
# 256 where its uint8 digits break): transforms from the CPU backend,
# balls from the brute-force backend
WIDE_CELLS = [
    ("torus_linf", [250, 240], 1, 1), ("torus_linf", [250, 240], 2, 1),
    ("grid_linf", [250, 240], 1, 1), ("torus_linf", [33, 40, 17], 1, 1),
]


def sha(a, dtype):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()
                          ).hexdigest()


def key(*parts):
    return "__".join(str(p) for p in parts)


def cell_id(problem, axes, R, mu):
    return f"{problem}-{'x'.join(map(str, axes))}-R{R}-mu{mu}"


def fields(b, code, out, pre):
    b.recount(code)
    out[key(pre, "cnt")] = b.read_cnt().astype(np.uint16)
    b.gain_map()
    out[key(pre, "gain")] = b.map.astype(np.int32).copy()
    b.loss_map()
    out[key(pre, "loss")] = b.map.astype(np.int32).copy()


def small(out, tables):
    t0 = time.time()
    # --- transform cells (multiset codes, like the reference's GPU test)
    for axes, R, mu in TRANSFORM_CELLS:
        cid = cell_id("hamming", axes, R, mu)
        c = NumpyDPBackend(axes, R, mu=mu)
        rng = np.random.default_rng(sum(axes) + R)
        size = c.space.size
        for k, m in enumerate((1, max(2, size // 50), max(3, size // 7))):
            code = rng.integers(0, size, size=m).astype(np.int64)
            out[key(cid, k, "code")] = code
            fields(c, code, out, key(cid, k))
    # --- family cells: fields, gathers, updates, queries
    for problem, axes, R, mu in FAMILY_CELLS + WIDE_CELLS:
        cid = cell_id(problem, axes, R, mu)
        c = NumpyDPBackend(axes, R, problem=problem, mu=mu)
        size = c.space.size
        wide = max(axes) > 16
        rng = np.random.default_rng(31)
        code = np.sort(rng.choice(size, size=max(2, size // 40),
                                  replace=False)).astype(np.int64)
        out[key(cid, "code")] = code
        fields(c, code, out, cid)
        probe = rng.integers(0, size, size=200).astype(np.int64)
        out[key(cid, "probe")] = probe
        c.recount(code)
        if wide:
            r = REF[problem](axes, R, mu=mu)
            r.recount(code)
            assert (r.cnt == c.cnt).all(), cid
            src = r
        else:
            src = c
        for t in (0, 1, 2):
            out[key(cid, "gather", t)] = src.ball_gather(probe, t)
        words, signs = update_sequence(size, code, 40, 7)
        out[key(cid, "upd_words")] = words
        out[key(cid, "upd_signs")] = signs
        for w, s in zip(words, signs):
            src.ball_update(np.array([w]), int(s))
        out[key(cid, "upd_cnt")] = src.read_cnt().astype(np.uint16)
        out[key(cid, "upd_gather0")] = src.ball_gather(probe, 0)
        out[key(cid, "upd_gather1")] = src.ball_gather(probe, 1)
        c.recount(code)
        c.gain_map()
        mx = c.map_max()
        out[key(cid, "gain_max")] = np.int64(mx)
        out[key(cid, "gain_hist")] = c.map_hist(16, max(mx, 1))
        thr = max(1, mx // 2)
        idx, val, found = c.map_extract(thr)
        out[key(cid, "ext_thr")] = np.int64(thr)
        out[key(cid, "ext_idx")] = idx
        out[key(cid, "ext_found")] = np.int64(found)
        out[key(cid, "deficit")] = np.int64(c.uncovered())
        out[key(cid, "count_eq")] = np.array(
            [c.count_eq(t) for t in range(4)], dtype=np.int64)
        # brute-force cross-check of the CPU backend's fields
        if size <= 1 << 16 and not wide:
            r = REF[problem](axes, R, mu=mu)
            r.recount(code)
            assert (r.cnt == c.cnt).all(), cid
            r.gain_map()
            assert (r.map == c.map).all(), cid
        if not wide:
            pats = support_patterns(axes, R, problem)
            tables[key(cid, "v1")] = pats
            tables[key(cid, "v1_local")] = locality_order(pats, axes)
    # --- K_3(8,2): 30 codewords (seed 0), 100 seeded updates
    cell = CELLS["K3_8_2"]
    c = NumpyDPBackend(list(cell.axes), cell.R)
    r = RefHammingBackend(list(cell.axes), cell.R)
    code = code_for(cell)
    out[key("K3_8_2", "code")] = code
    fields(c, code, out, "K3_8_2")
    c.recount(code)
    r.recount(code)
    words, signs = update_sequence(cell.size, code, 100, 100)
    out[key("K3_8_2", "upd_words")] = words
    out[key("K3_8_2", "upd_signs")] = signs
    trace_cnt, trace_q = [], []
    for w, s in zip(words, signs):
        c.ball_update(np.array([w]), int(s))
        r.ball_update(np.array([w]), int(s))
        assert (c.cnt == r.cnt).all()
        trace_cnt.append(c.read_cnt().astype(np.uint16))
        trace_q.append([c.count_eq(t) for t in range(4)] + [c.uncovered()])
    out[key("K3_8_2", "trace_cnt")] = np.stack(trace_cnt)
    out[key("K3_8_2", "trace_q")] = np.array(trace_q, dtype=np.int64)
    c.gain_map()
    out[key("K3_8_2", "upd_gain")] = c.map.astype(np.int32).copy()
    c.loss_map()
    out[key("K3_8_2", "upd_loss")] = c.map.astype(np.int32).copy()
    print(f"small fixtures: {len(out)} arrays in {time.time() - t0:.1f}s")


def full(path):
    res = {}
    for name in ("H3_14_3", "LEE_7_8_4", "KING_2048", "H3_16_4", "H2_26_3"):
        cell = CELLS[name]
        t0 = time.time()
        c = NumpyDPBackend(list(cell.axes), cell.R, problem=cell.problem)
        code = code_for(cell)
        d = {"M": int(cell.M), "code_sha": sha(code, "<i8")}
        c.recount(code)
        d["cnt_sha"] = sha(c.cnt, "<u2")
        d["count_eq"] = [c.count_eq(t) for t in range(4)]
        d["deficit"] = c.uncovered()
        d["cnt_max"] = int(c.cnt.max())
        c.gain_map()
        d["gain_sha"] = sha(c.map, "<i4")
        d["gain_max"] = c.map_max()
        d["gain_hist_sha"] = sha(c.map_hist(1024, max(1, c.map_max())),
                                 "<i4")
        c.loss_map()
        d["loss_sha"] = sha(c.map, "<i4")
        d["loss_at_code_sha"] = sha(c.map_read_at(code), "<i4")
        if cell.problem == "hamming":
            words, signs = update_sequence(cell.size, code, 1000, 1000)
            for w, s in zip(words, signs):
                c.ball_update(np.array([w]), int(s))
            d["upd_cnt_sha"] = sha(c.cnt, "<u2")
            d["upd_deficit"] = c.uncovered()
            c.gain_map()
            d["upd_gain_sha"] = sha(c.map, "<i4")
        if cell.problem == "lee":
            c.recount(code)
            cand = candidates(cell.size, 100000, 2000)
            d["cand_sha"] = sha(cand, "<i8")
            for t in (0, 1):
                d[f"gather{t}_sha"] = sha(c.ball_gather(cand, t), "<i4")
        d["seconds"] = round(time.time() - t0, 1)
        res[name] = d
        print(name, d, flush=True)
        with open(path, "w") as f:
            json.dump(res, f, indent=1, sort_keys=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--full", action="store_true")
    ap.add_argument("--only-full", action="store_true")
    args = ap.parse_args()
    if not args.only_full:
        out, tables = {}, {}
        small(out, tables)
        np.savez_compressed(os.path.join(HERE, "small_fields.npz"), **out)
        np.savez_compressed(os.path.join(HERE, "support_tables.npz"),
                            **tables)
    if args.full or args.only_full:
        full(os.path.join(HERE, "full_configs.json"))


if __name__ == "__main__":
    main()
