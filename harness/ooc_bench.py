"""Streamed (out-of-HBM) transforms against the host link.

A cell whose layer planes do not fit the device budget keeps them in
pinned host memory and streams them through device pieces in two phases
(``coldcore_b200.outofcore``).  This leg times coverage transforms (code
-> cnt) of binary Hamming n=30, R=3 (2^30 words: 8.6 GB of 16-bit host
planes) with the device budget forced to 8 GB, and measures the host link
itself (pinned 1 GB copies each way) as the bound: each live plane crosses
the link once per phase, so the transform's link bytes over the slower
direction's copy rate is its floor.  The reference's comparison point is
its K_10(10,5) whole-space transform over GH200's C2C link, 73-110 s
(``docs/benchmarks.md:53-65``); its link bytes at this leg's measured rate
are reported as a projection.

    python -m harness.ooc_bench [--axes 2x30 --R 3 --budget-gb 8]
"""
import argparse
import json
from math import prod

import numpy as np


def link_rates(nbytes=1 << 30, reps=3):
    """Pinned host <-> device copy GB/s (best of reps) each way."""
    import torch
    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    out = {}
    for name, dst, src in (("h2d", d, h), ("d2h", h, d)):
        best = None
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            dst.copy_(src, non_blocking=True)
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        out[name] = round(nbytes / best / 1e6, 2)
    del h, d
    return out


# the reference's K_10(10,5): (R+1) = 6 planes of 10^10 words at 2 bytes,
# each crossing the link once a phase (two phases)
K10_LINK_BYTES = 2 * 6 * 10 ** 10 * 2


def link_projection_s(link_bytes, best_ms, target_bytes=K10_LINK_BYTES):
    """Seconds that `target_bytes` of link traffic take at the rate a
    transform achieved (`link_bytes` crossed in `best_ms` milliseconds)."""
    return target_bytes / (link_bytes / (best_ms * 1e-3))


def measure(axes=None, R=3, budget_gb=8.0, code_words=100000, reps=3):
    import torch
    from coldcore_b200.outofcore import ooc_plan, ooc_transform
    axes = axes or [2] * 30
    X = prod(axes)
    rng = np.random.default_rng(1)
    code = np.unique(rng.integers(0, X, code_words))
    budget = int(budget_gb * 2 ** 30)
    plan = ooc_plan("hamming", axes, R, 0, 2, budget, M=len(code),
                    maxmult=1)
    rates = link_rates()
    host = torch.empty(plan["host_bytes"], dtype=torch.uint8,
                       pin_memory=True)
    times = []
    for _ in range(reps):
        _, ms = ooc_transform("hamming", axes, R, 0, 2, budget, code=code,
                              host=host)
        times.append([round(ms[0], 3), round(ms[1], 3)])
    best = min(t[0] + t[1] for t in times)
    # phase 1 is device-to-host bound, phase 2 host-to-device bound
    half = plan["link_bytes"] / 2
    floor_ms = half / (rates["d2h"] * 1e6) + half / (rates["h2d"] * 1e6)
    return {"cell": f"binary Hamming n={len(axes)}, R={R}", "words": X,
            "device_budget_GB": budget_gb, "code_words": int(len(code)),
            "plan": {k: plan[k] for k in ("split", "n_slabs", "n_cols",
                                          "host_bytes", "device_bytes",
                                          "link_bytes")},
            "phase_ms": times, "best_ms": round(best, 3),
            "link_GBps": round(plan["link_bytes"] / best / 1e6, 2),
            "link_measured_GBps": rates,
            "link_floor_ms": round(floor_ms, 3),
            "frac_of_link_floor": round(floor_ms / best, 3),
            # the K_10(10,5) link bytes at this leg's achieved link rate
            "projection_K10_10_5_s": round(
                link_projection_s(plan["link_bytes"], best), 2),
            "reference_K10_10_5_s": "73-110 (GH200, C2C)"}


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--axes", default="2x30")
    ap.add_argument("--R", type=int, default=3)
    ap.add_argument("--budget-gb", type=float, default=8.0)
    a = ap.parse_args()
    q, n = (int(v) for v in a.axes.split("x"))
    print(json.dumps(measure([q] * n, a.R, a.budget_gb), indent=1))


if __name__ == "__main__":
    main()
