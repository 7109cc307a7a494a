"""Seeded synthetic workloads: the cells the engine is measured and
parity-checked on, and their codes, update sequences and candidate sets.

Every draw comes from ``np.random.default_rng(seed)``; codes are drawn with
``rng.choice(|X|, M, replace=False)`` (distinct codewords).  "~60% coverage"
means ``M = floor(-ln(0.4) |X| / |B|)``, "3% density" ``M = floor(0.03 |X|)``.
"""
import math
from dataclasses import dataclass, field

import numpy as np


@dataclass(frozen=True)
class Cell:
    name: str
    problem: str
    axes: tuple
    R: int
    M: int
    seed: int
    mu: int = 1
    extra: dict = field(default_factory=dict, compare=False, hash=False)

    @property
    def size(self):
        return int(np.prod(np.asarray(self.axes, dtype=np.int64)))


def cover_size(size, ball, frac):
    """Codewords of a uniform random code expected to cover ``frac``."""
    return int(math.floor(-math.log(1.0 - frac) * size / ball))


# ball cardinalities of the named cells
_B_H2_26_3 = 1 + 26 + 325 + 2600          # sum_{r<=3} C(26,r)
_B_H3_16_4 = sum(math.comb(16, r) * 2 ** r for r in range(5))
_B_H3_14_3 = sum(math.comb(14, r) * 2 ** r for r in range(4))

CELLS = {
    # the reference's CPU-runnable case: K_3(8,2), 30 codewords, seed 0
    "K3_8_2": Cell("K3_8_2", "hamming", (3,) * 8, 2, 30, 0),
    # large single-instance transforms (~60% coverage)
    "H2_26_3": Cell("H2_26_3", "hamming", (2,) * 26, 3,
                    cover_size(2 ** 26, _B_H2_26_3, 0.6), 1),
    "H3_16_4": Cell("H3_16_4", "hamming", (3,) * 16, 4,
                    cover_size(3 ** 16, _B_H3_16_4, 0.6), 2),
    # non-Hamming plugins at 3% density
    "LEE_7_8_4": Cell("LEE_7_8_4", "lee", (7,) * 8, 4,
                      int(0.03 * 7 ** 8), 3),
    "KING_2048": Cell("KING_2048", "torus_linf", (2048, 2048), 1,
                      int(0.03 * 2048 * 2048), 4),
    # the learned-LNS cell
    "H3_14_3": Cell("H3_14_3", "hamming", (3,) * 14, 3,
                    cover_size(3 ** 14, _B_H3_14_3, 0.6), 5),
    # the cell of coldcore's published update / gather latencies (K_8(9,4)
    # with 940 codewords; |B| = 333,166), here a seeded random code
    "K8_9_4": Cell("K8_9_4", "hamming", (8,) * 9, 4, 940, 6),
}


def code_for(cell):
    rng = np.random.default_rng(cell.seed)
    return np.sort(rng.choice(cell.size, size=cell.M, replace=False)
                   ).astype(np.int64)


def update_sequence(size, code, n, seed):
    """``n`` single-word updates: with probability 1/2 add a uniformly
    random non-member, else remove a uniformly random member.  Returns
    (words int64[n], signs int8[n])."""
    rng = np.random.default_rng(seed)
    live = [int(w) for w in code]
    members = set(live)
    words = np.empty(n, dtype=np.int64)
    signs = np.empty(n, dtype=np.int8)
    for i in range(n):
        if rng.random() < 0.5 or not live:
            w = int(rng.integers(size))
            while w in members:
                w = int(rng.integers(size))
            live.append(w)
            members.add(w)
            words[i], signs[i] = w, 1
        else:
            k = int(rng.integers(len(live)))
            w = live[k]
            live[k] = live[-1]
            live.pop()
            members.discard(w)
            words[i], signs[i] = w, -1
    return words, signs


def candidates(size, n, seed):
    """``n`` uniformly random candidate words (repeats allowed)."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, size, size=n).astype(np.int64)


def batch_cells(count=256, seed=7, lo=3.0, hi=7.0):
    """The batched-campaign workload: ``count`` seeded cells of uneven size.

    q uniform in {2..6}; n = round(log_q(10^U[lo, hi])) (so q^n is
    log-uniform in 10^lo..10^hi); R uniform in {1..4}, clipped to n;
    Hamming with probability 0.8, else Lee; a uniform random code covering
    about half the space (M = floor(ln 2 |X| / |B|), at least 1).
    Returns a list of (problem, axes, R, code)."""
    from .patterns import ball_size
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        q = int(rng.integers(2, 7))
        n = max(1, int(round(rng.uniform(lo, hi) * math.log(10) / math.log(q))))
        R = min(int(rng.integers(1, 5)), n)
        problem = "hamming" if rng.random() < 0.8 else "lee"
        axes = (q,) * n
        size = q ** n
        ball = ball_size(axes, R, problem)
        M = max(1, min(size, int(math.floor(math.log(2.0) * size / ball))))
        code = np.sort(rng.choice(size, size=M, replace=False)).astype(np.int64)
        out.append((problem, axes, R, code))
    return out
