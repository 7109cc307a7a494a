"""Replica plumbing for multi-GPU runs: one process per GPU, each working
on its own cell (the transform has no exchange-free split, so ranks are
replicas).  ``torch.distributed`` carries only the barrier and the
reductions of timings: NCCL when the ranks have GPUs, gloo otherwise.

Ranks read RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* from the environment
(torchrun).  The process group gets a short timeout, so ranks that wait
for a rank that died end with an error instead of hanging.
"""
import datetime
import os


class ReplicaGroup:
    def __init__(self, backend=None, timeout_s=120):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.backend = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(
                backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.pg = dist
            self.backend = backend

    def _reduce(self, v, op):
        if not self.pg:
            return v
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(v)], device=dev, dtype=torch.float64)
        self.pg.all_reduce(t, op=op)
        return float(t.item())

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v):
        """The largest value over ranks (the job's time is its slowest)."""
        return self._reduce(v, self.pg.ReduceOp.MAX if self.pg else None)

    def sum(self, v):
        return self._reduce(v, self.pg.ReduceOp.SUM if self.pg else None)

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()
            self.pg = None


def aggregate_rate(units_per_rank, ms_max, world):
    """Whole-job throughput: all ranks' units over the slowest rank's
    time (weak scaling, one replica per rank)."""
    return units_per_rank * world / (ms_max * 1e-3)
