"""The batched engine's per-cell calls and the campaign driver on a B200:
per-cell codes, updates, gathers, counts and map queries against the
oracle; a campaign of searches in lock step whose every cover the oracle
verifies, beside the same jobs on one singleton context per cell."""
import numpy as np
import pytest

from coldcore_b200.batch import BatchEngine
from coldcore_b200.campaign import run_campaign, run_serial
from coldcore_b200.patterns import wide_table
from oracle.dp_oracle import OracleBackend

pytestmark = pytest.mark.gpu

CELLS = [("hamming", (3,) * 7, 2, 1), ("lee", (5,) * 5, 2, 1),
         ("hamming", (2,) * 12, 2, 2), ("torus_linf", (7, 8, 9), 1, 1),
         ("hamming", (2,) * 18, 3, 1)]


def test_per_cell_calls_match_the_oracle():
    rng = np.random.default_rng(3)
    with BatchEngine() as b:
        for p, a, R, mu in CELLS:
            b.add(p, a, R, np.zeros(0, dtype=np.int64), mu)
        b.build(0)
        oracles = []
        for k, (p, a, R, mu) in enumerate(CELLS):
            b.set_table(k, wide_table(a, R, p))
            size = int(np.prod(a))
            code = np.sort(rng.choice(size, max(2, size // 50),
                                      replace=False))
            b.set_code(k, code)
            o = OracleBackend(list(a), R, problem=p, mu=mu)
            o.recount(code)
            oracles.append(o)
        for rnd in range(2):
            b.run(0)
            for k, (p, a, R, mu) in enumerate(CELLS):
                o, size = oracles[k], int(np.prod(a))
                assert np.array_equal(b.cnt(k), o.read_cnt()), (rnd, k)
                o.gain_map()
                assert np.array_equal(b.gain(k), o.map), (rnd, k)
                idx = rng.integers(0, size, 97)
                assert np.array_equal(b.read_at(k, 1, idx), o.map[idx])
                thr = max(1, int(o.map.max()) // 2)
                ei, ev, found = b.extract(k, 1, thr, 1 << 16)
                want = np.flatnonzero(o.map >= thr)
                assert found == len(want)
                assert np.array_equal(np.sort(ei), want)
                # updates (three words added, then taken back) and
                # gathers of every role on the updated counters
                drop = np.unique(rng.integers(0, size, 3))
                b.update(k, drop, +1)
                o.ball_update(drop, +1)
                assert np.array_equal(b.cnt(k), o.read_cnt())
                assert b.count(k, 0, 0) == o.count_eq(0)
                assert b.count(k, 1) == o.uncovered()
                probe = rng.integers(0, size, 123)
                for role in (0, 1, 2):
                    assert np.array_equal(b.gather(k, probe, role),
                                          o.ball_gather(probe, role))
                b.update(k, drop, -1)
                o.ball_update(drop, -1)
                # a new code for the next launch
                newc = np.sort(rng.choice(size, max(2, size // 40),
                                          replace=False))
                b.set_code(k, newc)
                o.recount(newc)


def test_campaign_covers_verify_and_match_the_serial_arm():
    jobs = [{"problem": p, "axes": list(a), "R": R, "mu": mu, "seed": 5 + k,
             "budget_s": 60.0}
            for k, (p, a, R, mu) in enumerate(CELLS)]
    jobs.append({"problem": "hamming", "axes": [3] * 6, "R": 1, "seed": 9,
                 "mode": "descend", "budget_s": 8.0, "notch_s": 2.0})
    recs, ticks = run_campaign(jobs)
    serial = run_serial(jobs)
    assert ticks > 0
    for j, r, sr in zip(jobs, recs, serial):
        assert r["error"] is None, r["error"]
        assert r["uncov"] == 0
        o = OracleBackend(j["axes"], j["R"], problem=j["problem"],
                          mu=j.get("mu", 1))
        o.recount(np.asarray(r["code"], np.int64))
        assert o.uncovered() == 0 and len(r["code"]) == r["M"]
        # same algorithm and seed; extraction order may differ on a GPU
        assert sr["uncov"] == 0
        assert abs(r["M"] - sr["M"]) <= max(3, sr["M"] // 20), (r, sr)


def test_batched_device_repair_equals_the_singleton_repair():
    """repair="device": the batched greedy (one launch per step for every
    cell) places exactly the words the singleton's device greedy places,
    so both campaigns end in the same covers, word for word."""
    jobs = [{"problem": p, "axes": list(a), "R": R, "mu": mu, "seed": 11 + k,
             "budget_s": 60.0, "repair": "device"}
            for k, (p, a, R, mu) in enumerate(CELLS)]
    recs, ticks = run_campaign(jobs)
    serial = run_serial(jobs)
    for j, r, sr in zip(jobs, recs, serial):
        assert r["error"] is None and sr["error"] is None, (r, sr)
        assert r["uncov"] == 0 == sr["uncov"]
        assert r["code"] == sr["code"], j
        o = OracleBackend(j["axes"], j["R"], problem=j["problem"],
                          mu=j.get("mu", 1))
        o.recount(np.asarray(r["code"], np.int64))
        assert o.uncovered() == 0
