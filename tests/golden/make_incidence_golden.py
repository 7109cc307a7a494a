"""Generate ``incidence_golden.npz``: the reference's own explicit-incidence
backends (coldcore ``src/coldcore/incidence.py``) run on seeded inputs.

Needs the reference source tree, with ``COLDCORE_REF_SRC`` naming its
``src/`` directory:

    python tests/golden/make_incidence_golden.py

Cells:
  * dense random incidences, the shapes of the reference's own parity
    cases (``tests/test_incidence.py:64``), mu 1 and 2;
  * covering-design incidences C(v,k,t) built by the reference's
    ``problems.covering_design.build_incidence`` (blocks and t-subsets by
    colex rank);
  * weighted CSR incidences (variable row lengths, some empty, w in 1..3,
    uw in 1..4), mu 1..3.

Each cell records three rounds of: a seeded solution, its recount (cnt,
uncovered, count_eq 0..3), the gain and loss maps, gathers at 21 probe
candidates for targets 0, 1, 2, 5, then seven additions and three
removals and the cnt after them.
"""
import os
import sys

import numpy as np

REF_SRC = os.environ.get("COLDCORE_REF_SRC")
if not REF_SRC or not os.path.isdir(os.path.join(REF_SRC, "coldcore")):
    sys.exit("set COLDCORE_REF_SRC to the reference checkout's src/ "
             "directory (the one holding the coldcore package)")
sys.path.insert(0, REF_SRC)

from coldcore.incidence import (SparseIncidenceBackend,  # noqa: E402
                                WeightedIncidenceBackend)
from coldcore.problems.covering_design import (all_blocks,  # noqa: E402
                                               build_incidence)

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "incidence_golden.npz")

DENSE = [(60, 4, 40, 1), (120, 7, 80, 2), (25, 3, 9, 1), (200, 10, 300, 2),
         (90, 33, 120, 1), (40, 1, 12, 3)]
DESIGNS = [(9, 4, 2, 1), (13, 4, 2, 1), (10, 5, 3, 2), (8, 4, 3, 1)]
WEIGHTED = [(50, 30, 1, 7), (80, 45, 2, 8), (120, 60, 3, 9), (33, 20, 2, 10)]


def random_incidence(rng, n_cand, d, n_univ):
    return np.stack([np.sort(rng.choice(n_univ, d, replace=False))
                     for _ in range(n_cand)]).astype(np.int32)


def random_csr(rng, n_cand, n_univ):
    lens = rng.integers(0, 9, n_cand)
    lens[rng.choice(n_cand, max(1, n_cand // 10), replace=False)] = 0
    indptr = np.concatenate(([0], np.cumsum(lens))).astype(np.int64)
    indices = np.concatenate(
        [np.sort(rng.choice(n_univ, int(m), replace=False)) for m in lens]
        or [np.zeros(0)]).astype(np.int32)
    w = rng.integers(1, 4, len(indices)).astype(np.int32)
    uw = rng.integers(1, 5, n_univ).astype(np.int32)
    return indptr, indices, w, uw


def record(out, key, backend, n_cand, rng):
    for r in range(3):
        M = int(rng.integers(0, n_cand // 2 + 1))
        sol = np.sort(rng.choice(n_cand, M, replace=False)).astype(np.int64)
        backend.recount(sol)
        p = f"{key}/{r}/"
        out[p + "sol"] = sol
        out[p + "cnt"] = backend.cnt.astype(np.int32).copy()
        out[p + "uncovered"] = np.int64(backend.uncovered())
        out[p + "count_eq"] = np.array([backend.count_eq(t) for t in range(4)],
                                       dtype=np.int64)
        backend.gain_map()
        out[p + "gain"] = backend.map.astype(np.int32).copy()
        backend.loss_map()
        out[p + "loss"] = backend.map.astype(np.int32).copy()
        probe = rng.choice(n_cand, 21).astype(np.int64)
        out[p + "probe"] = probe
        for t in (0, 1, 2, 5):
            out[p + f"gather{t}"] = backend.ball_gather(probe, t).astype(
                np.int32)
        add = rng.choice(n_cand, 7).astype(np.int64)
        out[p + "add"] = add
        backend.ball_update(add, +1)
        backend.ball_update(add[:3], -1)
        out[p + "upd_cnt"] = backend.cnt.astype(np.int32).copy()


def main():
    out = {}
    for i, (n_cand, d, n_univ, mu) in enumerate(DENSE):
        rng = np.random.default_rng(1000 + i)
        inc = random_incidence(rng, n_cand, d, n_univ)
        key = f"dense{i}"
        out[key + "/inc"] = inc
        out[key + "/meta"] = np.array([n_univ, mu], dtype=np.int64)
        record(out, key, SparseIncidenceBackend(inc, n_univ, mu=mu), n_cand,
               rng)
    for i, (v, k, t, mu) in enumerate(DESIGNS):
        rng = np.random.default_rng(2000 + i)
        inc = build_incidence(all_blocks(v, k), v, t)
        n_univ = int(inc.max()) + 1
        key = f"design{i}"
        out[key + "/inc"] = inc
        out[key + "/meta"] = np.array([n_univ, mu, v, k, t], dtype=np.int64)
        record(out, key, SparseIncidenceBackend(inc, n_univ, mu=mu),
               len(inc), rng)
    for i, (n_cand, n_univ, mu, seed) in enumerate(WEIGHTED):
        rng = np.random.default_rng(3000 + seed)
        indptr, indices, w, uw = random_csr(rng, n_cand, n_univ)
        key = f"weighted{i}"
        out[key + "/indptr"] = indptr
        out[key + "/indices"] = indices
        out[key + "/w"] = w
        out[key + "/uw"] = uw
        out[key + "/meta"] = np.array([n_univ, mu], dtype=np.int64)
        record(out, key, WeightedIncidenceBackend(indptr, indices, w, n_univ,
                                                  uw=uw, mu=mu), n_cand, rng)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(out)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
