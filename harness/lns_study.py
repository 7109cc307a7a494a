"""Time-to-size study of the learned ruin proposal against plain LNS.

    python -m harness.lns_study --q 3 --n 14 --R 3 --seeds 5 \
        --budget 120 --moves 100000 --out study.json

Steps, all on the GPU engine:

1. **Start.** For each evaluation seed, a greedy start: ``load([])``, the
   exact greedy from empty, then ``peel``.
2. **Log.** Plain LNS descents (fixed mix) on separate training seeds, with
   :class:`~coldcore_b200.learned.MoveLog` attached, until ``--moves``
   removals are logged.
3. **Train.** :func:`~coldcore_b200.learned.train_scorer` on the log.  The
   AUC on held-out rounds is reported, pooled and within rounds.
4. **Evaluate.** From each seed's greedy start, a ``budget``-second notch
   descent with ``select="fixed"``, ``"adaptive"`` and ``"learned"``.
   Each run records the wall time at which each verified size was reached.
   The target of a seed is the best size either plain run reached.  The
   metric is the learned run's wall time to that size, divided by the
   faster plain run's time to it.
"""
import argparse
import json
import sys
import time

import numpy as np

from coldcore_b200.learned import (LearnedRuin, MoveLog, RuinFeatures,
                                   train_scorer)
from coldcore_b200.search import Searcher


def greedy_start(b, seed):
    s = Searcher(b, seed=seed)
    s.build_reserve_s = 0.0
    s.load([])
    s.greedy_fill(10 ** 9)
    s.peel()
    if s.verify_full() != 0:
        raise RuntimeError("greedy start is not a cover")
    return s.code.copy()


def descent(b, start, seed, budget, select, proposer=None, move_log=None,
            notch_s=10.0, kmin=8, kmax=None, step0=4, repair="exact"):
    """One timed notch descent; returns ([(seconds, M), ...], stats, ok)
    with the verified sizes in the order they were reached."""
    t0 = time.time()
    trace = []
    s = Searcher(b, seed=seed, deadline=t0 + budget, proposer=proposer,
                 move_log=move_log, repair=repair,
                 on_solved=lambda m, c: trace.append(
                     (round(time.time() - t0, 3), int(m))))
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load(start)
    s.descend(notch_budget_s=notch_s, step0=step0, reserve_s=0.0,
              min_notch_s=1.0, kmin=kmin, kmax=kmax, select=select,
              fail_limit=10 ** 6)
    # descend reports a size only after a full recount; check the last too
    ok = s.verify_full() == 0
    return trace, s.stats, ok


def time_to(trace, size):
    for t, m in trace:
        if m <= size:
            return t
    return None


def log_moves(b, feats, moves, budget, notch_s, kmin=8, kmax=None,
              seed0=1000, say=print, repair="exact"):
    """Plain (fixed-mix) descents on seeds seed0, seed0 + 1, ... with the
    move log attached, until ``moves`` removals or ``budget`` seconds."""
    t0 = time.time()
    mlog = MoveLog(feats, cap=moves)
    seed = seed0
    while not mlog.full and time.time() - t0 < budget:
        start = greedy_start(b, seed)
        left = budget - (time.time() - t0)
        s = Searcher(b, seed=seed, deadline=time.time() + min(left, 120.0),
                     move_log=mlog, repair=repair)
        s.build_reserve_s = s.loop_reserve_s = 0.0
        s.load(start)
        s.descend(notch_budget_s=notch_s, step0=4, reserve_s=0.0,
                  min_notch_s=1.0, kmin=kmin, kmax=kmax, fail_limit=10 ** 6)
        say(f"log seed {seed}: {len(mlog)} moves, {mlog.rounds} rounds, "
            f"{time.time() - t0:.0f}s")
        seed += 1
    return mlog


class LossScorer:
    """Ablation scorer: the negative z-scored exact loss.  The proposer
    then draws like a ``low`` ruin through the same Gumbel top-k rule, so
    the gap to the MLP scorer is what the model adds over the pick rule."""

    heldout_auc = None

    def __call__(self, X):
        lo = np.asarray(X, dtype=np.float64)[:, 0]
        return -(lo - lo.mean()) / (lo.std() + 1e-12)


def evaluate(b, feats, scorer, seeds, budget, notch_s, selects, kmin=8,
             kmax=None, say=print, repair="exact", **learned_kw):
    """``selects``: any of "fixed", "adaptive", "learned" and "loss-topk"
    (the ablation: the learned proposer driven by :class:`LossScorer`)."""
    runs = []
    for seed in seeds:
        start = greedy_start(b, seed)
        row = {"seed": seed, "start_M": int(len(start))}
        for sel in selects:
            prop = None
            if sel in ("learned", "loss-topk"):
                prop = LearnedRuin(scorer if sel == "learned" else
                                   LossScorer(), feats, seed=seed,
                                   **learned_kw)
            fsec0 = feats.seconds
            trace, stats, ok = descent(b, start, seed, budget,
                                       "learned" if prop else sel,
                                       proposer=prop, notch_s=notch_s,
                                       kmin=kmin, kmax=kmax, repair=repair)
            row[sel] = {"trace": trace, "ok": ok,
                        "best": trace[-1][1] if trace else None,
                        "rounds": stats["rounds"],
                        "learned_rounds": stats["learned_rounds"],
                        "fallback_rounds": stats["fallback_rounds"],
                        "feature_s": round(feats.seconds - fsec0, 2)}
            if prop is not None:
                row[sel]["gate"] = dict(prop.stats)
            say(f"seed {seed} {sel}: best {row[sel]['best']} "
                f"rounds {stats['rounds']} ok {ok}")
        plain = [s for s in ("fixed", "adaptive") if s in row]
        if plain and "learned" in row:
            row.update(time_to_size(row, plain, budget))
            say(f"seed {seed}: target {row['target_M']} plain "
                f"{row['t_plain']}s learned {row['t_learned']}s")
        runs.append(row)
    return runs


def time_to_size(row, plain, budget):
    """The target is the best size the plain arms reached, and at least one
    word below the start.  ratio = learned time to it / plain time to it.
    When no plain arm reached it within the budget, the plain time is
    above the budget and ratio_bound = learned time / budget bounds the
    ratio from above."""
    target = min([row[s]["best"] for s in plain] + [row["start_M"] - 1])
    tps = [t for t in (time_to(row[s]["trace"], target) for s in plain)
           if t is not None]
    tp = min(tps) if tps else None
    tl = time_to(row["learned"]["trace"], target)
    out = {"target_M": target, "t_plain": tp, "t_learned": tl,
           "ratio": (tl / tp) if (tl is not None and tp) else None,
           "ratio_bound": None}
    if tp is None and tl is not None:
        out["ratio_bound"] = tl / budget
    return out


def summarize(runs):
    """Per-seed ratios; a seed where only the learned arm reached the
    target counts with its upper bound, one where neither did is left out.
    Also the best sizes of each arm."""
    rows = [r for r in runs if "target_M" in r]
    vals = []
    for r in rows:
        v = r["ratio"] if r["ratio"] is not None else r["ratio_bound"]
        if v is not None:
            vals.append(v)
    out = {"seeds": len(rows), "learned_reached": f"{len(vals)}/{len(rows)}",
           "median_ratio": float(np.median(vals)) if vals else None,
           "geo_mean_ratio": (float(np.exp(np.mean(np.log(vals))))
                              if vals else None),
           "ratios": [round(v, 3) for v in vals]}
    for arm in ("fixed", "adaptive", "learned", "loss-topk"):
        bests = [r[arm]["best"] for r in runs if arm in r]
        if bests:
            out[f"best_{arm}"] = bests
    return out


def main(argv=None):
    from coldcore_b200.gpu import GpuBackend
    ap = argparse.ArgumentParser()
    ap.add_argument("--q", type=int, default=3)
    ap.add_argument("--n", type=int, default=14)
    ap.add_argument("--R", type=int, default=3)
    ap.add_argument("--seeds", type=int, default=5)
    ap.add_argument("--budget", type=float, default=120.0)
    ap.add_argument("--notch", type=float, default=10.0)
    ap.add_argument("--kmin", type=int, default=8)
    ap.add_argument("--kmax", type=int, default=None)
    ap.add_argument("--moves", type=int, default=100000)
    ap.add_argument("--log-budget", type=float, default=600.0)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--selects", default="fixed,adaptive,learned")
    ap.add_argument("--temperature", type=float, default=0.5)
    ap.add_argument("--pick", default="topk", choices=("topk", "anchor"))
    ap.add_argument("--scale", default="raw", choices=("raw", "std"))
    ap.add_argument("--repair", default="exact", choices=("exact", "device"),
                    help="LNS repair of every arm: the Python lazy greedy "
                         "(the reference's) or the device exact greedy")
    ap.add_argument("--out", default=None)
    ap.add_argument("--save-log", default=None)
    ap.add_argument("--load-log", default=None)
    a = ap.parse_args(argv)

    def say(*x):
        print(*x, file=sys.stderr, flush=True)

    b = GpuBackend([a.q] * a.n, a.R, "hamming")
    feats = RuinFeatures(b)
    report = {"cell": f"K_{a.q}({a.n},{a.R})", "budget_s": a.budget,
              "notch_s": a.notch, "kmin": a.kmin, "kmax": a.kmax,
              "temperature": a.temperature, "pick": a.pick,
              "scale": a.scale,
              "repair": a.repair}
    t0 = time.time()
    if a.load_log:
        z = np.load(a.load_log)
        X, y, g = z["X"], z["y"], z["g"]
    else:
        mlog = log_moves(b, feats, a.moves, a.log_budget, a.notch,
                         kmin=a.kmin, kmax=a.kmax, say=say, repair=a.repair)
        X, y, g = mlog.arrays()
        if a.save_log:
            np.savez_compressed(a.save_log, X=X, y=y, g=g)
    report["log"] = {"moves": int(len(y)), "rounds": int(len(np.unique(g))),
                     "positive": float(y.mean()) if len(y) else 0.0,
                     "seconds": round(time.time() - t0, 1)}
    say("log", report["log"])
    t1 = time.time()
    scorer = train_scorer(X, y, g, epochs=a.epochs)
    report["train"] = {"heldout_auc": scorer.heldout_auc,
                       "heldout_within_round_auc": scorer.within_auc,
                       "train_auc": scorer.train_auc,
                       "seconds": round(time.time() - t1, 2)}
    say("train", report["train"])
    runs = evaluate(b, feats, scorer, range(1, a.seeds + 1), a.budget,
                    a.notch, a.selects.split(","), kmin=a.kmin, kmax=a.kmax,
                    say=say, repair=a.repair, temperature=a.temperature,
                    pick=a.pick, scale=a.scale)
    report["runs"] = runs
    report["summary"] = summarize(runs)
    say("summary", report["summary"])
    b.close()
    if a.out:
        with open(a.out, "w") as f:
            json.dump(report, f)
    print(json.dumps(report["summary"]))
    return report


if __name__ == "__main__":
    main()
