"""The campaign driver's lock-step ticks and its per-cell protocol adapter,
on the host: a stand-in batch whose cells are the numpy oracle.  Every
search must end in a cover the oracle verifies, the ticks must batch the
searches' transforms, and a failing search must become an error record
without stalling the others."""
import numpy as np

from coldcore_b200.campaign import run_campaign
from oracle.dp_oracle import OracleBackend


class OracleBatch:
    """BatchEngine's interface over one OracleBackend per cell."""

    def __init__(self, fail_cell=None):
        self.cells, self.runs, self.fail_cell = [], 0, fail_cell

    def add(self, problem, axes, R, code, mu=1):
        o = OracleBackend(list(axes), R, problem=problem, mu=mu)
        o.recount(np.asarray(code, dtype=np.int64))
        self.cells.append({"o": o, "code": np.asarray(code, np.int64),
                           "gain": None, "loss": None})
        return len(self.cells) - 1

    def build(self, tile_kb=0):
        pass

    def set_table(self, cell, tbl):
        assert tbl.ndim == 2 and len(tbl) >= 1

    def set_code(self, cell, code):
        self.cells[cell]["code"] = np.asarray(code, np.int64)

    def run(self, mode=0):
        self.runs += 1
        for c in self.cells:
            o = c["o"]
            o.recount(c["code"])
            o.gain_map()
            c["gain"] = o.map.copy()
            o.loss_map()
            c["loss"] = o.map.copy()

    def scalars(self):
        return np.array([[c["o"].uncovered(), c["gain"].max(initial=0),
                          c["loss"].max(initial=0)] for c in self.cells],
                        dtype=np.int64)

    def update(self, cell, words, delta):
        if cell == self.fail_cell:
            raise RuntimeError("planted failure")
        self.cells[cell]["o"].ball_update(words, delta)

    def gather(self, cell, words, role):
        return self.cells[cell]["o"].ball_gather(words, role)

    def greedy(self, cells, adds):
        from oracle.dp_oracle import exact_greedy
        out = []
        for k, add in zip(cells, adds):
            c = self.cells[k]
            out.append(exact_greedy(c["o"], c["code"], add))
        return out

    def count(self, cell, mode, target=0):
        o = self.cells[cell]["o"]
        return o.uncovered() if mode == 1 else o.count_eq(target)

    def _map(self, cell, field):
        return self.cells[cell]["gain" if field == 1 else "loss"]

    def extract(self, cell, field, thr, cap):
        m = self._map(cell, field)
        idx = np.flatnonzero(m >= thr)
        return idx[:cap].astype(np.int64), m[idx[:cap]].astype(np.int32), \
            len(idx)

    def read_at(self, cell, field, idx):
        return self._map(cell, field)[np.asarray(idx, np.int64)].astype(
            np.int32)

    def read_range(self, cell, field, off, length):
        return self.cells[cell]["o"].read_cnt(off, length)

    def close(self):
        pass


JOBS = [{"problem": "hamming", "axes": [3] * 5, "R": 1, "seed": 1},
        {"problem": "hamming", "axes": [2] * 8, "R": 1, "seed": 2},
        {"problem": "lee", "axes": [5, 5, 5], "R": 1, "seed": 3},
        {"problem": "hamming", "axes": [3] * 4, "R": 1, "mu": 2, "seed": 4}]


def test_campaign_searches_verify_on_the_oracle():
    eng = OracleBatch()
    recs, ticks = run_campaign(JOBS, engine=eng)
    assert ticks == eng.runs and ticks > 0
    for j, r in zip(JOBS, recs):
        assert r["error"] is None, r["error"]
        assert r["uncov"] == 0 and r["M"] == len(r["code"])
        o = OracleBackend(j["axes"], j["R"], problem=j["problem"],
                          mu=j.get("mu", 1))
        o.recount(np.asarray(r["code"], np.int64))
        assert o.uncovered() == 0
    # the searches ran in lock step: far fewer ticks than transforms
    transforms = sum(r["stats"]["transforms"] for r in recs)
    assert ticks < transforms


def test_a_failing_search_is_recorded_and_the_others_finish():
    recs, _ = run_campaign(JOBS[:3], engine=OracleBatch(fail_cell=1))
    assert recs[1]["error"] and "planted failure" in recs[1]["error"]
    assert recs[0]["uncov"] == 0 and recs[2]["uncov"] == 0


def test_device_repair_runs_in_the_ticks():
    """repair="device": every search's greedy runs inside a tick, batched
    with the others, and ends in the same cover as the exact greedy."""
    jobs = [dict(j, repair="device") for j in JOBS]
    eng = OracleBatch()
    recs, ticks = run_campaign(jobs, engine=eng)
    for j, r in zip(jobs, recs):
        assert r["error"] is None, r["error"]
        assert r["uncov"] == 0
        o = OracleBackend(j["axes"], j["R"], problem=j["problem"],
                          mu=j.get("mu", 1))
        o.recount(np.asarray(r["code"], np.int64))
        assert o.uncovered() == 0
