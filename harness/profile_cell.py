"""Run one cell's transforms a few times — a small, fixed workload for
``ncu`` captures and ``DCT_TIMING=1`` per-launch timings.

    python -m harness.profile_cell --cell H2_26_3 --mode gain --reps 2

Prints the launch plan (first axis, axes, algorithmic bytes, kernel id) and,
with --timing, each launch's device milliseconds and GB/s.
"""
import argparse

from coldcore_b200.gpu import GpuBackend
from coldcore_b200.workloads import CELLS, code_for

MODES = {"recount": (0, 2), "gain": (1, 1), "loss": (2, 1)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cell", default="H2_26_3", choices=sorted(CELLS))
    ap.add_argument("--mode", default="gain", choices=sorted(MODES) + ["all"])
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--timing", action="store_true")
    ap.add_argument("--nvtx", action="store_true",
                    help="after the timed reps (and the autotuner), run one "
                         "more transform per mode inside an NVTX range "
                         "named 'capture' (ncu --nvtx --nvtx-include "
                         "capture/ then sees the tuned launches only)")
    args = ap.parse_args()
    cell = CELLS[args.cell]
    modes = list(MODES) if args.mode == "all" else [args.mode]
    with GpuBackend(list(cell.axes), cell.R, problem=cell.problem) as b:
        b.recount(code_for(cell))
        b.set_timing(args.timing)
        for m in modes:
            i, o = MODES[m]
            for _ in range(args.reps):
                if b._lib.dct_transform(i, o):
                    raise RuntimeError("transform failed")
            plan = b.plan(i, o)              # after the autotuner ran
            print(f"{cell.name} {m}: plan (axis0, axes, bytes, kernel) = "
                  f"{plan.tolist()}, forms (1 pipe, 2 pack, 4 in16, "
                  f"8 out16, 16 pair) = {b.plan_forms(i, o).tolist()}")
            if args.nvtx:
                import torch
                torch.cuda.nvtx.range_push("capture")
                if b._lib.dct_transform(i, o):
                    raise RuntimeError("transform failed")
                torch.cuda.synchronize()
                torch.cuda.nvtx.range_pop()
            if args.timing:
                for k, t in enumerate(b.last_timings()):
                    by = int(plan[k][2])
                    print(f"  launch {k}: {t:.4f} ms  {by / t / 1e6:.1f} GB/s")


if __name__ == "__main__":
    main()
