"""A fixed workload for ncu captures of the batched step: the 256-cell
campaign (``workloads.batch_cells(256, seed=7)``) built on one BatchEngine,
two steps, then one step inside the NVTX range ``capture`` (so that
``ncu --nvtx --nvtx-include capture/`` sees one step's launches only).

    python -m harness.batch_profile
"""
import torch

from coldcore_b200.batch import BatchEngine
from coldcore_b200.workloads import batch_cells


def main():
    cells = batch_cells(256, seed=7)
    with BatchEngine() as b:
        for p, a, R, code in cells:
            b.add(p, a, R, code)
        b.build(0)
        for _ in range(2):
            b.run(0)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("capture")
        b.run(0)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    print("ok")


if __name__ == "__main__":
    main()
