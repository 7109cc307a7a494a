"""Field throughput of the explicit-incidence engine on a covering design.

One step = a gain field and a loss field over every candidate of C(v,k,t)
(default C(30,8,4): 5,852,925 blocks x 70 triples, a 1.64 GB incidence,
27,405 universe elements) after a recount of a seeded solution, the
incidence built on the device.  Reported per field: milliseconds, and GB/s
of its algorithmic bytes (the incidence read once, the map written once,
cnt read once).  Given another ABI-2 library (``--ref PATH``, e.g. the
reference's own ``src/plugins/sparse/sparse.cu`` built for sm_100a), its
kernels are timed in alternation on the same incidence.

    python -m harness.incidence_bench [--v 30 --k 8 --t 4 --reps 20]
                                            [--ref PATH] [--bits]

The default row form tests one role bit per universe element in shared
memory; ``--bits`` also times the counter form (``CC_SPARSE_BITS=0``: one
counter read per row entry) and checks its gain field against the default
form's (reported under ``counter_form``).
"""
import argparse
import json
import os
import statistics
import time

import numpy as np


def _warm(b, seconds=0.3):
    """Fields until `seconds` have passed: clocks settle before timing."""
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        b.gain_map()
        b.loss_map()


def _time_fields(b, stream, reps):
    """Mean ms of gain + loss fields, CUDA events on `stream`."""
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        b.gain_map()
        b.loss_map()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / (2 * reps)


def measure(v=30, k=8, t=4, reps=20, rounds=3, ref_path=None,
            cpu_field=None, bits=False):
    """Both cells stay resident and are timed in alternation, `rounds`
    times each after a warm-up; the medians are reported.  ``cpu_field``
    (optional, the caller's CPU baseline): ``cpu_field(rows, cnt, out)``
    computes the gain field of the host copy of the incidence; it is
    timed over three calls and checked against the engine's field."""
    import torch

    from coldcore_b200.incidence import (GpuCoveringDesignBackend,
                                         GpuIncidenceBackend)
    rng = np.random.default_rng(v * 100 + k * 10 + t)
    out = {"design": f"C({v},{k},{t})"}
    with GpuCoveringDesignBackend(v, k, t) as b:
        n_cand, d, n_univ = b.n_cand, b.d, b.n_univ
        sol = rng.choice(n_cand, max(1, n_cand // 2000), replace=False)
        b.recount(sol)
        stream = torch.cuda.ExternalStream(int(b._lib.sparse_b200_stream()))
        host_rows = b.rows()
        host_cnt = b.read_cnt().astype(np.int32)
        ref = None
        if ref_path:
            ref = GpuIncidenceBackend(host_rows, n_univ, plugin_path=ref_path)
        try:
            if ref is not None:
                ref.recount(sol)
                _warm(ref)
            _warm(b)
            ours, theirs = [], []
            for _ in range(rounds):
                ours.append(_time_fields(b, stream, reps))
                if ref is not None:
                    theirs.append(_time_fields(ref, torch.cuda.default_stream(),
                                               reps))
            # the same engine with one CTA wave per SM instead of four
            os.environ["CC_SPARSE_BLOCKS_PER_SM"] = "8"
            try:
                _warm(b, 0.1)
                one_wave = [_time_fields(b, stream, reps)
                            for _ in range(rounds)]
            finally:
                os.environ.pop("CC_SPARSE_BLOCKS_PER_SM", None)
            b.gain_map()
            sample = np.arange(0, n_cand, 997)
            gain = b.map_read_at(sample)
            bit_rounds = bits_same = None
            if bits:
                # the other row form: a counter read per row entry
                os.environ["CC_SPARSE_BITS"] = "0"
                try:
                    _warm(b, 0.1)
                    bit_rounds = [_time_fields(b, stream, reps)
                                  for _ in range(rounds)]
                    b.gain_map()
                    bits_same = bool(np.array_equal(b.map_read_at(sample),
                                                    gain))
                finally:
                    os.environ.pop("CC_SPARSE_BITS", None)
            same = None
            if ref is not None:
                ref.gain_map()
                same = bool(np.array_equal(ref.map_read_at(sample), gain))
        finally:
            if ref is not None:
                ref.close()
    cpu_ms = cpu_same = None
    if cpu_field is not None:
        out_map = np.empty(n_cand, dtype=np.int32)
        cpu_field(host_rows, host_cnt, out_map)
        t0 = time.perf_counter()
        for _ in range(3):
            cpu_field(host_rows, host_cnt, out_map)
        cpu_ms = (time.perf_counter() - t0) / 3 * 1e3
        cpu_same = bool(np.array_equal(out_map[sample], gain))
    ms = statistics.median(ours)
    by = n_cand * (d + 1) * 4 + n_univ * 4
    out.update({"n_cand": n_cand, "d": d, "n_univ": n_univ,
                "incidence_gb": round(n_cand * d * 4 / 1e9, 3),
                "solution": len(sol), "ms_per_field": round(ms, 4),
                "ms_rounds": [round(x, 4) for x in ours],
                "ms_rounds_8_ctas_per_sm": [round(x, 4) for x in one_wave],
                "GBps": round(by / (ms * 1e-3) / 1e9, 1),
                "algorithmic_bytes_per_field": by})
    if bit_rounds is not None:
        bms = statistics.median(bit_rounds)
        out["counter_form"] = {"ms_per_field": round(bms, 4),
                            "ms_rounds": [round(x, 4) for x in bit_rounds],
                            "GBps": round(by / (bms * 1e-3) / 1e9, 1),
                            "same_gain_sample": bits_same}
    if cpu_ms is not None:
        out["cpu_baseline"] = {
            "value": round(by / (cpu_ms * 1e-3) / 1e9, 2), "unit": "GB/s",
            "cores": os.cpu_count(), "kind": "port",
            "sample": f"3 gain fields of {out['design']}, C restatement on "
                      f"all host threads, {cpu_ms:.1f} ms each",
            "same_gain_sample": cpu_same}
    if theirs:
        rms = statistics.median(theirs)
        out["reference_plugin"] = {
            "library": os.path.basename(ref_path),
            "ms_per_field": round(rms, 4),
            "ms_rounds": [round(x, 4) for x in theirs],
            "GBps": round(by / (rms * 1e-3) / 1e9, 1),
            "same_gain_sample": same,
            "speedup": round(rms / ms, 2)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--v", type=int, default=30)
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--t", type=int, default=4)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--ref", default=None,
                    help="another ABI-2 library to time beside the engine")
    ap.add_argument("--bits", action="store_true",
                    help="also time the counter form (CC_SPARSE_BITS=0)")
    a = ap.parse_args()
    print(json.dumps(measure(a.v, a.k, a.t, a.reps, ref_path=a.ref,
                             bits=a.bits)))


if __name__ == "__main__":
    main()
