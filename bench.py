#!/usr/bin/env python3
"""Transform throughput of the B200 covering engine on its headline cell.

A STEP is the three whole-space transforms of one cell — recount (code ->
cnt), gain map and loss map — through the plugin ABI.  The headline cell is
binary Hamming n=26, R=3 (|X| = 67.1M, the larger of the two large
single-instance cells; 20,830 seeded codewords, ~60% coverage); ternary
n=16, R=4 is measured after it and reported under "also".

value : model GB/s (the one-axis-per-pass byte model, the same for every
        implementation, coldcore_b200.metrics) with the code resident on
        the device; CUDA events on the engine's stream; inputs (1.07 GB of
        layers) are larger than the 126 MB L2.
e2e   : the same metric through the public C-ABI with host buffers: every
        step uploads the code from host memory (dct_set_code) and reads
        three scalars back (uncovered count, two map maxima).
roofline : the dominant launch: its algorithmic bytes (cnt / layers read,
        layers / map / cnt written, from the engine's own launch plan) over
        its mean CUDA-event duration, against the measured HBM copy peak.
cpu_baseline : the C restatement of the reference's CPU axis DP on every
        host thread (oracle/cport), a bounded sample of the same cell.

lns   : (1 GPU) LNS time-to-verified-size on K_3(14,3), learned ruin
        proposal against plain LNS from the same greedy start, five seeds
        (1..5; the moves for training are logged on seeds 1000..), median
        and geometric mean of the per-seed time ratios.

--impl reference runs that CPU restatement alone (rank 0), on the same
cell, metric and unit: each step one transform of the cell, rotating
recount / gain / loss.  When the reference's own plugin has been built for
sm_100a (oracle/build_ref.py) and a GPU is present, that arm also times it
on the cells it accepts (H3_16_4, K_3(14,3), K_3(8,2)) under "gpu_plugin";
the B200 arm reports the engine on the same cells under "same_cells".

Multi-GPU (torchrun): every rank runs its own replica of the cell (the
transform does not shard into independent pieces without an exchange
step); value is the sum over ranks of the model bytes over the max time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from coldcore_b200.metrics import model_bytes          # noqa: E402
from coldcore_b200.replicas import ReplicaGroup         # noqa: E402
from coldcore_b200.workloads import CELLS, code_for     # noqa: E402

METRIC = ("transform GB/s vs HBM peak; LNS time-to-verified-size learned "
          "vs plain, 1 B200")
HEADLINE = "H2_26_3"
ALSO = "H3_16_4"


def step_model_bytes(cell):
    ax, R, p = list(cell.axes), cell.R, cell.problem
    return (model_bytes(ax, R, p, "recount") + model_bytes(ax, R, p, "gain")
            + model_bytes(ax, R, p, "loss"))


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel_key):
    """Per-launch DRAM bytes from a committed ncu summary, if present."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(kernel_key)
    except Exception:
        return None


# ---------------------------------------------------------------- dist
class Dist(ReplicaGroup):
    """The bench's replica group (``coldcore_b200.replicas``)."""


# ---------------------------------------------------------------- clocks
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            return None
        return parse_clock_samples(out)


def parse_clock_samples(text):
    """nvidia-smi samples (the Clocks.FIELDS columns, csv, no header, no
    units) -> median SM clock, max clock and every throttle reason seen
    active; None without a usable sample."""
    sm, mx, reasons = [], None, set()
    names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
             "sw_power_cap")
    for line in text.strip().splitlines():
        f = [x.strip() for x in line.split(",")]
        if len(f) < 9:
            continue
        try:
            sm.append(float(f[1]))
            mx = float(f[2])
        except ValueError:
            continue
        for k, name in enumerate(names):
            if f[5 + k].lower().startswith("active"):
                reasons.add(name)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
            "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- CPU arm
def cpu_sample(cell, modes, code):
    """Model GB/s of the C restatement over the given transforms."""
    from oracle.cport import CPortCell
    c = CPortCell(list(cell.axes), cell.R, cell.problem)
    c.recount(code)
    by, t = 0, 0.0
    for m in modes:
        t0 = time.perf_counter()
        if m == "recount":
            c.recount(code)
        elif m == "gain":
            c.gain_map()
        else:
            c.loss_map()
        t += time.perf_counter() - t0
        by += model_bytes(list(cell.axes), cell.R, cell.problem, m)
    return by / t / 1e9, t


def ref_plugin_gpu(args):
    """The reference's own ABI-v1 plugin, compiled from its source for
    sm_100a (oracle/build_ref.py), timed on this B200 over the cells it
    accepts (axes <= 16, n <= 16, <= 65,535 occurrences): one step =
    recount + gain map + loss map, CUDA events on the default stream the
    plugin uses.  None when the library or the GPU is absent."""
    path = os.path.join(ROOT, "oracle", "_ref", "libref_covering.so")
    if not os.path.exists(path):
        return None
    import torch
    if not torch.cuda.is_available():
        return None
    from coldcore_b200.gpu import GpuBackend
    out = {"library": "oracle/_ref/libref_covering.so (reference "
                      "src/plugins/covering/dct_hc.cu, nvcc -O3 sm_100a)"}
    for name in ("H3_16_4", "H3_14_3", "K3_8_2"):
        cell = CELLS[name]
        code = code_for(cell)
        with GpuBackend(list(cell.axes), cell.R, problem=cell.problem,
                        plugin_path=path) as b:
            lib = b._lib
            b._set_code(code)

            def step():                   # the B200 arm's step, same calls
                if lib.dct_transform(0, 2) or lib.dct_transform(1, 1) or \
                        lib.dct_transform(2, 1):
                    raise RuntimeError("reference transform failed")
            for _ in range(args.warmup):
                step()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            reps = max(3, args.steps // 2)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(reps):
                step()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
        by = sum(model_bytes(list(cell.axes), cell.R, cell.problem, m)
                 for m in ("recount", "gain", "loss"))
        out[name] = {"ms_per_step": round(ms, 4),
                     "value": round(by / (ms * 1e-3) / 1e9, 1),
                     "unit": "GB/s"}
    return out


def run_reference(args, dist):
    if dist.rank != 0:
        return
    cell = CELLS[args.cell]
    code = code_for(cell)
    from oracle.cport import CPortCell, build
    build()
    c = CPortCell(list(cell.axes), cell.R, cell.problem)
    c.recount(code)
    modes = ("recount", "gain", "loss")
    fns = {"recount": lambda: c.recount(code), "gain": c.gain_map,
           "loss": c.loss_map}
    for i in range(args.warmup):
        fns[modes[i % 3]]()
    by, t = 0, 0.0
    for i in range(args.steps):
        m = modes[i % 3]
        t0 = time.perf_counter()
        fns[m]()
        t += time.perf_counter() - t0
        by += model_bytes(list(cell.axes), cell.R, cell.problem, m)
    val = by / t / 1e9
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 3),
        "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * t / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic",
        "config": {"workload": cell.name, "axes": f"{cell.axes[0]}^"
                   f"{len(cell.axes)}", "R": cell.R, "M": cell.M,
                   "step": "one transform (recount / gain / loss, rotating)",
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": round(val, 3), "unit": "GB/s",
                         "cores": cores, "kind": "port",
                         "sample": f"{args.steps} transforms of {cell.name} "
                                   "(C restatement, OpenMP, all threads)"},
        "e2e": {"value": round(val, 3), "unit": "GB/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_ref_gpu:
        gp = ref_plugin_gpu(args)
        if gp:
            line["gpu_plugin"] = gp
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm
def measure_cell(cell, args, dist, timed=True):
    import torch

    from coldcore_b200.gpu import GpuBackend
    code = code_for(cell)
    b = GpuBackend(list(cell.axes), cell.R, problem=cell.problem)
    stream = torch.cuda.ExternalStream(b.stream)
    lib = b._lib
    res = {}
    try:
        b._set_code(code)

        def step():
            if lib.dct_transform(0, 2) or lib.dct_transform(1, 1) or \
                    lib.dct_transform(2, 1):
                raise RuntimeError("transform failed")

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        dist.barrier()
        clocks = Clocks(dist.local)
        if timed:
            clocks.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("timed")     # ncu --nvtx-include timed/
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        dist.barrier()
        ms = dist.max(e0.elapsed_time(e1)) / args.steps
        res["clocks"] = clocks.stop() if timed else None
        res["ms"] = ms
        if timed:
            # the same steps back to back for at least a second, with its
            # own clock record: shows the K-step number is the steady one
            reps = max(args.steps, int(1.2e3 / max(ms, 1e-3)) + 1)
            sclk = Clocks(dist.local)
            sclk.start()
            dist.barrier()
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(reps):
                step()
            e1.record(stream)
            torch.cuda.synchronize()
            dist.barrier()
            sms = dist.max(e0.elapsed_time(e1))
            res["sustained"] = {"steps": reps, "seconds": round(sms / 1e3, 3),
                                "ms_per_step": round(sms / reps, 4),
                                "clocks": sclk.stop()}
        res["value"] = step_model_bytes(cell) * dist.world / (ms * 1e-3) / 1e9
        res["launches_per_step"] = sum(
            len(b.plan(i, o)) for i, o in ((0, 2), (1, 1), (2, 1)))

        # ---- e2e through the public API with host buffers
        host_code = np.ascontiguousarray(code)

        def step_e2e():
            b.recount(host_code)
            u = b.uncovered()
            b.gain_map()
            m1 = b.map_max()
            b.loss_map()
            m2 = b.map_max()
            return u, m1, m2

        for _ in range(max(1, args.warmup // 2)):
            step_e2e()
        torch.cuda.synchronize()
        dist.barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        f0.record(stream)
        for _ in range(args.steps):
            step_e2e()
        f1.record(stream)
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) * 1e3 / args.steps
        ms_e2e = dist.max(max(wall, f0.elapsed_time(f1) / args.steps))
        res["e2e"] = {
            "value": round(step_model_bytes(cell) * dist.world
                           / (ms_e2e * 1e-3) / 1e9, 3),
            "unit": "GB/s", "ms_per_step": round(ms_e2e, 4),
            "h2d_bytes_per_step": int(code.nbytes),
            "d2h_bytes_per_step": 24}

        # ---- per-launch timing for the roofline (separate pass)
        b.set_timing(True)
        b._set_code(code)
        per = {}
        for _ in range(max(3, args.steps // 2)):
            for (i, o) in ((0, 2), (1, 1), (2, 1)):
                if lib.dct_transform(i, o):
                    raise RuntimeError("transform failed")
                plan = b.plan(i, o)
                for k, t in enumerate(b.last_timings()):
                    per.setdefault((i, o, k), []).append(t)
        b.set_timing(False)
        rows = []
        for (i, o, k), ts in per.items():
            plan = b.plan(i, o)
            forms = b.plan_forms(i, o)
            j0, nax, by, kid = (int(v) for v in plan[k])
            mean = sum(ts) / len(ts)
            rows.append({"transform": f"({i},{o})", "launch": k,
                         "axes": f"{j0}..{j0 + nax - 1}", "kernel_id": kid,
                         "form": form_name(forms[k] if k < len(forms) else 0),
                         "bytes": by, "ms": mean,
                         "GBps": by / (mean * 1e-3) / 1e9})
        res["launches"] = rows
        return res
    finally:
        b.close()


def step_rate(out):
    """A batched step's achieved DRAM-side rate: its algorithmic bytes (each
    launch's source read once, its destination written once; the batch
    plan's own count) over the persistent step time, against the peak."""
    peak, peak_kind = peaks()
    gbs = out["step_bytes"] / (out["persistent"]["ms_per_step"] * 1e-3) / 1e9
    return {"step_GBps": round(gbs, 1), "step_frac": round(gbs / peak, 4),
            "peak_kind": peak_kind}


def measure_batch_small(args):
    """A campaign of many small cells, where a persistent launch pays:
    1,024 seeded cells of 10^3..10^5 words (otherwise as measure_batch).
    Persistent graph launch against one launch per pass per cell."""
    import torch

    from coldcore_b200.batch import BatchEngine
    from coldcore_b200.workloads import batch_cells
    cells = batch_cells(1024, seed=11, lo=3.0, hi=5.0)
    out = {"cells": len(cells),
           "words": int(sum(int(np.prod(a)) for _, a, _, _ in cells))}
    with BatchEngine() as b:
        for p, a, R, code in cells:
            b.add(p, a, R, code)
        b.build(0)
        out["step_bytes"] = b.info()["step_bytes"]
        for mode, key in ((0, "persistent"), (1, "per_pass_launches")):
            for _ in range(2):
                b.run(mode)
            torch.cuda.synchronize()
            reps = max(3, args.steps // 4)
            t0 = time.perf_counter()
            for _ in range(reps):
                b.run(mode)
            dt = (time.perf_counter() - t0) / reps
            out[key] = {"ms_per_step": round(1e3 * dt, 3),
                        "instances_per_s": round(len(cells) / dt, 1)}
    out["speedup"] = round(out["persistent"]["instances_per_s"]
                           / out["per_pass_launches"]["instances_per_s"], 2)
    out.update(step_rate(out))
    if not args.no_cpu:
        from oracle.cport import campaign_rate     # the CPU baseline leg
        rate, wall, busy, workers = campaign_rate(cells)
        out["cpu_baseline"] = {
            "value": round(rate, 2), "unit": "instances/s", "cores": workers,
            "kind": "port",
            "sample": f"all {len(cells)} cells, one step each, C restatement, "
                      f"{workers} single-threaded spawned worker processes: "
                      f"{wall:.1f} s wall, {busy:.1f} s busy"}
        out["speedup_vs_cpu"] = round(
            out["persistent"]["instances_per_s"] / rate, 1)
    return out


def form_name(f):
    """Schedule form flags of one launch (GpuBackend.plan_forms) as text."""
    names = [("pipe", 1), ("pack", 2), ("in16", 4), ("out16", 8),
             ("pair", 16), ("tma", 32), ("u8", 64)]
    return "+".join(n for n, bit in names if int(f) & bit) or "plain"


def measure_batch(args, dist):
    """Batched campaign: 256 seeded cells of uneven size (q in 2..6, q^n
    log-uniform in 10^3..10^7, R in 1..4, 80% Hamming / 20% Lee, codes
    covering ~half of each space).  One step = every cell's recount,
    deficit, gain map + max, loss map + max.  Persistent graph launch
    against one launch per pass per cell (same engine)."""
    import torch

    from coldcore_b200.batch import BatchEngine
    from coldcore_b200.workloads import batch_cells
    cells = batch_cells(256, seed=7)
    out = {}
    with BatchEngine() as b:
        for p, a, R, code in cells:
            b.add(p, a, R, code)
        t0 = time.perf_counter()
        b.build(0)
        out["build_s"] = round(time.perf_counter() - t0, 2)
        out.update(b.info())
        for mode, key in ((0, "persistent"), (1, "per_pass_launches")):
            for _ in range(2):
                b.run(mode)
            torch.cuda.synchronize()
            reps = max(3, args.steps // 4)
            t0 = time.perf_counter()
            for _ in range(reps):
                b.run(mode)
            dt = (time.perf_counter() - t0) / reps
            out[key] = {"ms_per_step": round(1e3 * dt, 3),
                        "instances_per_s": round(len(cells) / dt, 1)}
    # the campaign as coldcore runs it: one singleton cell context per
    # instance (init, code upload, three transforms, two scalars, free)
    from coldcore_b200.gpu import GpuBackend
    t0 = time.perf_counter()
    for p, a, R, code in cells:
        with GpuBackend(list(a), R, problem=p) as g:
            g.recount(code)
            g.uncovered()
            g.gain_map()
            g.map_max()
            g.loss_map()
            g.map_max()
    dt = time.perf_counter() - t0
    out["singleton_per_cell"] = {"ms_per_step": round(1e3 * dt, 3),
                                 "instances_per_s": round(len(cells) / dt, 1)}
    out["speedup"] = round(out["persistent"]["instances_per_s"]
                           / out["per_pass_launches"]["instances_per_s"], 2)
    out["speedup_vs_singleton"] = round(
        out["persistent"]["instances_per_s"]
        / out["singleton_per_cell"]["instances_per_s"], 2)
    out.update(step_rate(out))
    out["words"] = int(sum(int(np.prod(a)) for _, a, _, _ in cells))
    if not args.no_cpu and dist.world == 1:
        # the reference campaign's own parallelism: one cell per process on
        # every host core, here with the C restatement of its CPU DP
        from oracle.cport import campaign_rate
        rate, wall, busy, workers = campaign_rate(cells)
        out["cpu_baseline"] = {
            "value": round(rate, 2), "unit": "instances/s", "cores": workers,
            "kind": "port",
            "sample": f"all {len(cells)} cells, one step each (recount, "
                      f"deficit, gain + max, loss + max), C restatement, "
                      f"{workers} single-threaded spawned worker processes, "
                      f"largest first: {wall:.1f} s wall, {busy:.1f} s busy"}
        out["speedup_vs_cpu"] = round(
            out["persistent"]["instances_per_s"] / rate, 1)
    return out


def measure_lns(args):
    """LNS time-to-verified-size on K_3(14,3) (4.78M words, R = 3) over
    several seeds: plain LNS moves are logged on other seeds and the MLP is
    trained on them; then, per seed, from one greedy start, a plain descent
    (record mix) and a learned-ruin descent run for the same wall-time
    budget.  A seed's ratio is the learned run's time to the plain run's
    best size over the plain run's time to it; reported with the median and
    the geometric mean over the seeds (harness.lns_study.summarize)."""
    from coldcore_b200.gpu import GpuBackend
    from coldcore_b200.learned import RuinFeatures, train_scorer
    from harness.lns_study import evaluate, log_moves, summarize
    t0 = time.perf_counter()
    seeds = list(range(1, args.lns_seeds + 1))
    with GpuBackend([3] * 14, 3) as b:
        feats = RuinFeatures(b)
        # the device exact greedy repairs every arm: plain LNS then makes
        # thousands of rounds a minute, so its time to its best size is
        # measured rather than bounded by the budget
        mlog = log_moves(b, feats, args.lns_moves, 120.0, 15.0,
                         say=lambda *a: None, repair="device")
        X, y, g = mlog.arrays()
        sc = train_scorer(X, y, g, epochs=15)
        runs = evaluate(b, feats, sc, seeds, args.lns_budget, 10.0,
                        ["fixed", "learned"], say=lambda *a: None,
                        repair="device")
    summ = summarize(runs)
    per_seed = [{"seed": r["seed"], "start_M": r["start_M"],
                 "target_M": r.get("target_M"),
                 "best_plain": r["fixed"]["best"],
                 "best_learned": r["learned"]["best"],
                 "t_plain_s": r.get("t_plain"),
                 "t_learned_s": r.get("t_learned"),
                 "ratio": r.get("ratio"), "ratio_bound": r.get("ratio_bound"),
                 "rounds_plain": r["fixed"]["rounds"],
                 "rounds_learned": r["learned"]["rounds"]} for r in runs]
    return {"cell": "K_3(14,3)", "seeds": seeds,
            "budget_s": args.lns_budget, "notch_s": 10.0,
            "repair": "device (both arms)",
            "median_ratio": summ["median_ratio"],
            "geo_mean_ratio": summ["geo_mean_ratio"],
            "learned_reached": summ["learned_reached"],
            "ratios": summ["ratios"],
            "learned_smaller_or_equal": sum(
                1 for r in per_seed
                if r["best_learned"] is not None and r["best_plain"] is not None
                and r["best_learned"] <= r["best_plain"]),
            "per_seed": per_seed,
            "moves_logged": int(len(y)), "heldout_auc": sc.heldout_auc,
            "wall_s": round(time.perf_counter() - t0, 1)}


def run_b200(args, dist):
    cell = CELLS[args.cell]
    res = measure_cell(cell, args, dist)
    also = None
    same = {}
    if not args.no_also and args.cell == HEADLINE:
        r2 = measure_cell(CELLS[ALSO], args, dist, timed=False)
        also = {"workload": ALSO, "value": round(r2["value"], 1),
                "ms_per_step": round(r2["ms"], 4),
                "e2e": r2["e2e"]["value"]}
        # the smaller cells the reference's own plugin also accepts
        for name in ("H3_14_3", "K3_8_2"):
            r3 = measure_cell(CELLS[name], args, dist, timed=False)
            same[name] = {"ms_per_step": round(r3["ms"], 4),
                          "value": round(r3["value"], 1)}
    if dist.rank != 0:
        return
    peak, peak_kind = peaks()
    rows = res["launches"]
    total = sum(r["ms"] for r in rows)
    dom = max(rows, key=lambda r: r["ms"])
    ach = dom["bytes"] / (dom["ms"] * 1e-3) / 1e9
    # the whole step's algorithmic bytes (every launch of the three fused
    # transforms) over the step time: the achieved DRAM-side rate
    step_bytes = sum(r["bytes"] for r in rows)
    step_rate = step_bytes / (res["ms"] * 1e-3) / 1e9
    # keyed by the launch's axes: the capture must be of the same group
    tkey = f"{cell.name}:{dom['transform']}:{dom['axes']}"
    traffic = ncu_traffic(tkey)
    cpu = None
    if dist.world == 1 and not args.no_cpu:
        code = code_for(cell)
        val, secs = cpu_sample(cell, ("recount", "gain", "loss"), code)
        cpu = {"value": round(val, 3), "unit": "GB/s",
               "cores": os.cpu_count(), "kind": "port",
               "sample": f"one step (recount + gain + loss) of {cell.name}, "
                         f"{secs:.1f} s, C restatement on all host threads"}
    line = {
        "metric": METRIC, "value": round(res["value"], 1), "unit": "GB/s",
        "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(res["ms"], 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic",
        "config": {
            "workload": cell.name, "axes": f"{cell.axes[0]}^{len(cell.axes)}",
            "R": cell.R, "M": cell.M, "seed": cell.seed,
            "step": "recount + gain map + loss map",
            "bytes_model": "one axis per pass (per-step model bytes "
                           f"{step_model_bytes(cell)})",
            "l2": "inputs larger than L2 (layers "
                  f"{(cell.R + 1) * cell.size * 4 / 1e9:.2f} GB)",
            "parallelism": f"replicas x{dist.world}",
            "launch_GBps": {f"{r['transform']}#{r['launch']}":
                            round(r["GBps"], 1) for r in rows},
            "launch_ms": {f"{r['transform']}#{r['launch']}":
                          round(r["ms"], 4) for r in rows},
            "launch_form": {f"{r['transform']}#{r['launch']}": r["form"]
                            for r in rows},
            "launch_axes": {f"{r['transform']}#{r['launch']}": r["axes"]
                            for r in rows},
        },
        "clocks": res["clocks"],
        "e2e": res["e2e"],
        "gpu_launches": res["launches_per_step"] * args.steps,
        "roofline": {"bound": "hbm", "achieved": round(ach, 1),
                     "peak": peak, "unit": "GB/s",
                     "frac": round(ach / peak, 4), "peak_kind": peak_kind,
                     "kernel": f"{dom['transform']} launch {dom['launch']} "
                               f"(axes {dom['axes']}, kernel id "
                               f"{dom['kernel_id']})",
                     "share": round(dom["ms"] / total, 3),
                     "algorithmic_bytes": dom["bytes"],
                     "traffic": traffic},
        "cpu_baseline": cpu,
        "step_rate": {"algorithmic_bytes": step_bytes,
                      "GBps": round(step_rate, 1),
                      "frac": round(step_rate / peak, 4),
                      "note": "every launch's algorithmic bytes of one step "
                              "over ms_per_step; value is the one-axis-per-"
                              "pass model rate"},
        "sustained": res.get("sustained"),
    }
    if also:
        line["also"] = also
    if same:
        line["same_cells"] = same
    # the secondary legs, each reporting a failure in its own object: the
    # ones measured before first, then the newer ones, so that an error in
    # a later leg cannot cost an earlier one its numbers
    def leg(key, fn):
        try:
            line[key] = fn()
        except Exception as e:           # noqa: BLE001
            line[key] = {"error": f"{type(e).__name__}: {e}"}

    if not args.no_batch:
        leg("batched", lambda: measure_batch(args, dist))
    if not args.no_lns and dist.world == 1:
        leg("lns", lambda: measure_lns(args))
    if not args.no_batch:
        leg("batched_small", lambda: measure_batch_small(args))
    if not args.no_batch and dist.world == 1:
        # a campaign of searches on the batched engine against one
        # singleton context per cell
        def campaign():
            from harness.campaign_bench import measure as camp_measure
            return camp_measure()
        leg("campaign", campaign)
    if not args.no_ops and dist.world == 1:
        # updates, per-candidate gathers and the Lee / king fields
        def ops():
            from harness.ops_bench import measure as ops_measure
            return ops_measure(cpu=not args.no_cpu)
        leg("ops", ops)
    if not args.no_ooc and dist.world == 1:
        # a cell streamed through a forced 8 GB device budget
        def ooc():
            from harness.ooc_bench import measure as ooc_measure
            return ooc_measure()
        leg("out_of_hbm", ooc)
    if not args.no_incidence and dist.world == 1:
        # the explicit-incidence engine (plugin ABI 2) on a covering design
        def incidence():
            from harness.incidence_bench import measure as inc_measure
            cpu_field = None
            if not args.no_cpu:
                from oracle.cport import inc_field

                def cpu_field(rows, cnt, out):     # the CPU baseline leg
                    inc_field(rows, cnt, 0, out=out)
            return inc_measure(cpu_field=cpu_field)
        leg("incidence", incidence)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--cell", default=HEADLINE, choices=sorted(CELLS))
    ap.add_argument("--no-also", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-incidence", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-lns", action="store_true")
    ap.add_argument("--no-ops", action="store_true")
    ap.add_argument("--no-ooc", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--lns-budget", type=float, default=30.0)
    ap.add_argument("--lns-seeds", type=int, default=5)
    ap.add_argument("--lns-moves", type=int, default=100000)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        # host-only arm: rank 0 measures, the other ranks exit without work
        if int(os.environ.get("RANK", "0")) == 0:
            run_reference(args, type("D", (), {"rank": 0})())
        return
    dist = Dist()
    try:
        run_b200(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
