"""Multi-process (world size 2, gloo, CPU) coverage of the replica plumbing
that the multi-GPU bench uses: barrier, max and sum over ranks, the
aggregate rate, and the reference arm under torchrun (rank 0 alone prints
one JSON line, the other rank exits without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from coldcore_b200.replicas import ReplicaGroup, aggregate_rate
    g = ReplicaGroup(backend="gloo", timeout_s=60)
    g.barrier()
    ms = 10.0 + 5.0 * rank                # rank 1 is the slow one
    mx = g.max(ms)
    sm = g.sum(rank + 1)
    rate = aggregate_rate(1000, mx, g.world)
    g.close()
    out.put((rank, g.backend, mx, sm, rate))


def test_replica_group_gloo_two_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, backend, mx, sm, rate in res:
        assert backend == "gloo"
        assert mx == 15.0                   # max over ranks
        assert sm == 3.0
        assert abs(rate - 1000 * 2 / 0.015) < 1e-6


def test_single_process_group_is_a_no_op(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from coldcore_b200.replicas import ReplicaGroup
    g = ReplicaGroup()
    assert g.world == 1 and g.max(3.5) == 3.5 and g.sum(2) == 2
    g.barrier()
    g.close()


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--cell", "K3_8_2",
           "--steps", "3", "--warmup", "3", "--no-ref-gpu"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=540,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1                  # rank 0 only
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0
