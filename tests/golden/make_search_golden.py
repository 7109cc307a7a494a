#!/usr/bin/env python3
"""Golden traces of the reference's search core on its own CPU backend.

Run in a checkout that has the reference source, with
``COLDCORE_REF_SRC`` naming its ``src/`` directory:

    python tests/golden/make_search_golden.py

For each small cell and seed it records, from ``coldcore.search.Searcher``
over ``coldcore.dp.NumpyDPBackend`` (whose ``map_extract`` returns
ascending indices, so a seeded run is deterministic):

* the code after ``load([])`` + ``greedy_fill`` from empty;
* the code after ``peel``;
* each ruin operator's removals from that code (``ruin(k, mode)``);
* the final code, uncovered count and round count of ``lns`` at one
  notch below the peeled size, with ``select="fixed"`` and
  ``"adaptive"`` (a run that does not solve within its 20 s budget is
  timing-dependent and is marked ``"solved": false``).

Output: ``search_traces.json`` (committed; nothing at test time reads the
reference).

With ``--deficit`` it writes ``search_deficit_traces.json`` instead: the
opt-in deficit-targeted ruin (``ruin(k, "deficit")`` after three ``low``
removals, so that words are uncovered) and ``lns(..., deficit=True)``
with both selections, from the same starting points.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SRC = os.environ.get("COLDCORE_REF_SRC")
if not REF_SRC or not os.path.isdir(os.path.join(REF_SRC, "coldcore")):
    sys.exit("set COLDCORE_REF_SRC to the reference checkout's src/ "
             "directory (the one holding the coldcore package)")
sys.path.insert(0, REF_SRC)

from coldcore.dp import NumpyDPBackend                       # noqa: E402
from coldcore.search import Searcher                          # noqa: E402

CELLS = [
    ("hamming", [3] * 6, 1, 1, 3),
    ("hamming", [2] * 9, 1, 1, 5),
    ("hamming", [4] * 4, 1, 1, 7),
    ("hamming", [3] * 5, 1, 2, 11),
    ("lee", [5, 5, 5], 1, 1, 13),
    ("hamming", [3, 4, 5], 1, 1, 17),
]


def backend(problem, axes, R, mu):
    return NumpyDPBackend(axes, R, problem=problem, mu=mu)


def built(problem, axes, R, mu, seed):
    s = Searcher(backend(problem, axes, R, mu), seed=seed)
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load([])
    s.greedy_fill(10 ** 9)
    return s


def main():
    out = []
    for problem, axes, R, mu, seed in CELLS:
        s = built(problem, axes, R, mu, seed)
        greedy = s.code.tolist()
        s.peel()
        peeled = s.code.tolist()
        assert s.verify_full() == 0
        ruins = {}
        for mode in ("low", "hole", "cluster", "random"):
            t = built(problem, axes, R, mu, seed)
            t.peel()
            removed = t.ruin(3, mode)
            ruins[mode] = {"removed": sorted(int(w) for w in removed),
                           "uncov": int(t.uncov)}
        lns = {}
        for select in ("fixed", "adaptive"):
            t = built(problem, axes, R, mu, seed)
            t.peel()
            M = len(t.code) - 1
            t.ruin(1, "low")
            unc = t.lns(M, round_budget_s=20.0, kmin=2, kmax=4,
                        select=select, log_every=0)
            lns[select] = {"M": M, "uncov": int(unc), "solved": unc == 0,
                           "rounds": int(t.stats["rounds"]),
                           "code": t.code.tolist()}
        out.append({"problem": problem, "axes": axes, "R": R, "mu": mu,
                    "seed": seed, "greedy": greedy, "peeled": peeled,
                    "ruin": ruins, "lns": lns})
        print(problem, axes, R, mu, "greedy", len(greedy), "peeled",
              len(peeled), {k: (v["uncov"], v["rounds"]) for k, v in
                            lns.items()}, flush=True)
    with open(os.path.join(HERE, "search_traces.json"), "w") as f:
        json.dump(out, f)


def main_deficit():
    out = []
    for problem, axes, R, mu, seed in CELLS:
        t = built(problem, axes, R, mu, seed)
        t.peel()
        t.ruin(3, "low")
        pre = t.uncovered_words().tolist()
        removed = t.ruin(3, "deficit")
        ruin = {"targets": [int(w) for w in pre],
                "removed": sorted(int(w) for w in removed),
                "uncov": int(t.uncov),
                "deficit_ruins": int(t.stats.get("deficit_ruins", 0))}
        lns = {}
        for select in ("fixed", "adaptive"):
            t = built(problem, axes, R, mu, seed)
            t.peel()
            M = len(t.code) - 1
            t.ruin(1, "low")
            unc = t.lns(M, round_budget_s=20.0, kmin=2, kmax=4,
                        select=select, log_every=0, deficit=True)
            lns[select] = {"M": M, "uncov": int(unc), "solved": unc == 0,
                           "rounds": int(t.stats["rounds"]),
                           "deficit_ruins": int(t.stats.get("deficit_ruins",
                                                            0)),
                           "code": t.code.tolist()}
        out.append({"problem": problem, "axes": axes, "R": R, "mu": mu,
                    "seed": seed, "ruin": ruin, "lns": lns})
        print(problem, axes, R, mu, ruin["removed"],
              {k: (v["uncov"], v["rounds"], v["deficit_ruins"])
               for k, v in lns.items()}, flush=True)
    with open(os.path.join(HERE, "search_deficit_traces.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    if "--deficit" in sys.argv:
        main_deficit()
    else:
        main()
