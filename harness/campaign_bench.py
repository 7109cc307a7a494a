"""A campaign of searches: the batched engine against one singleton context
per cell.

Jobs: ``workloads.batch_cells(count, seed, lo, hi)`` geometries (q in 2..6,
q^n log-uniform in 10^lo..10^hi words, R in 1..4, 80% Hamming / 20% Lee),
each job a greedy cover from empty followed by peel (a fixed amount of
search work, no time budget), the greedy on the device by default
(``repair="device"``: in the batched arm all cells' greedy steps share one
launch per step; in the serial arm each cell runs the singleton's device
greedy), or the Python lazy greedy (``--repair exact``).  The batched arm runs every job in lock step
on one BatchEngine (``coldcore_b200.campaign.run_campaign``); the serial
arm runs the same jobs one after another, each on its own singleton cell
context (``run_serial``), the pattern of coldcore's process-per-cell
campaign.  Reported: instances per second of each arm, the ticks, and how
many covers are complete.

    python -m harness.campaign_bench [--count 64 --lo 3 --hi 5]
"""
import argparse
import json
import time


def jobs_for(count=64, seed=13, lo=3.0, hi=5.0, repair="device"):
    from coldcore_b200.workloads import batch_cells
    return [{"problem": p, "axes": list(a), "R": R, "seed": 100 + k,
             "budget_s": 600.0, "mode": "build", "repair": repair}
            for k, (p, a, R, _code) in enumerate(
                batch_cells(count, seed=seed, lo=lo, hi=hi))]


def measure(count=64, seed=13, lo=3.0, hi=5.0, repair="device"):
    from coldcore_b200.campaign import run_campaign, run_serial
    jobs = jobs_for(count, seed, lo, hi, repair)
    run_campaign(jobs[:4])                  # warm the library and tables
    t0 = time.perf_counter()
    recs, ticks = run_campaign(jobs)
    tb = time.perf_counter() - t0
    t0 = time.perf_counter()
    srecs = run_serial(jobs)
    ts = time.perf_counter() - t0
    ok_b = sum(1 for r in recs if r["error"] is None and r["uncov"] == 0)
    ok_s = sum(1 for r in srecs if r["error"] is None and r["uncov"] == 0)
    same = sum(1 for r, q in zip(recs, srecs) if r.get("code") == q.get("code"))
    return {"jobs": len(jobs), "work": "greedy cover from empty + peel",
            "repair": repair, "identical_covers": same,
            "cells": f"batch_cells({count}, seed={seed}, lo={lo}, hi={hi})",
            "batched": {"seconds": round(tb, 3), "ticks": ticks,
                        "instances_per_s": round(len(jobs) / tb, 2),
                        "covers": ok_b,
                        "sum_M": int(sum(r["M"] or 0 for r in recs))},
            "serial_contexts": {"seconds": round(ts, 3),
                                "instances_per_s": round(len(jobs) / ts, 2),
                                "covers": ok_s,
                                "sum_M": int(sum(r["M"] or 0
                                                 for r in srecs))},
            "speedup": round(ts / tb, 2)}


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--count", type=int, default=64)
    ap.add_argument("--seed", type=int, default=13)
    ap.add_argument("--lo", type=float, default=3.0)
    ap.add_argument("--hi", type=float, default=5.0)
    ap.add_argument("--repair", default="device", choices=("device", "exact"))
    a = ap.parse_args()
    print(json.dumps(measure(a.count, a.seed, a.lo, a.hi, a.repair),
                     indent=1))


if __name__ == "__main__":
    main()
