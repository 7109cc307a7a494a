"""Support-table ("ball") builders for the engine.

The support set of a centre is its metric ball, enumerated as patterns of
(position, circular shift) pairs applied to the centre's digits — the
model of coldcore ``src/coldcore/patterns.py`` (v1 packed format, byte k =
``pos<<4 | delta``, entry 0 the centre).  Per-axis admissible shifts:

* ``hamming``: every shift 1..a-1, at most R positions changed;
* ``lee``: shifts of circular weight min(d, a-d) <= R, total weight <= R;
* ``torus_linf``: shifts within circular distance R, any positions;
* ``grid_linf``: the torus shifts (deduplicated when the window wraps);
  the device walk drops the ones that cross a board edge per centre.

Two encodings: the reference's packed v1 uint64 (axes <= 16, at most 8
changed positions) and this engine's wide table — ``slots`` int32 per
pattern, ``(pos << 24) | delta`` — which has no axis-width limit
(``dct_init3w``).
"""
from itertools import combinations

import numpy as np

PROBLEM_IDS = {"hamming": 0, "torus_linf": 1, "lee": 2, "grid_linf": 3}


def shift_sets(axes, R, problem):
    if problem == "hamming":
        return [np.arange(1, a, dtype=np.int64) for a in axes]
    if problem == "lee":
        return [np.array([d for d in range(1, a) if min(d, a - d) <= R],
                         dtype=np.int64) for a in axes]
    if problem in ("torus_linf", "grid_linf"):
        return [np.array(sorted({d for d in range(1, a)
                                 if d <= R or a - d <= R}), dtype=np.int64)
                for a in axes]
    raise ValueError(f"unknown problem {problem!r}")


def max_changed(n, R, problem):
    if problem in ("hamming", "lee"):
        return min(n, R)
    return n


def enumerate_ball(axes, R, problem):
    """(positions, deltas) arrays of shape (L, w); unused slots have delta
    0 and position 0.  Row 0 is the centre."""
    axes = [int(a) for a in axes]
    n = len(axes)
    sets = shift_sets(axes, R, problem)
    w = max(1, max_changed(n, R, problem))
    P = [np.zeros((1, w), dtype=np.int64)]
    D = [np.zeros((1, w), dtype=np.int64)]
    for k in range(1, max_changed(n, R, problem) + 1):
        for subs in combinations(range(n), k):
            parts = [sets[p] for p in subs]
            if any(len(s) == 0 for s in parts):
                continue
            mesh = np.meshgrid(*parts, indexing="ij")
            d = np.stack([m.ravel() for m in mesh], axis=1)
            if problem == "lee":
                wt = np.zeros(len(d), dtype=np.int64)
                for i, p in enumerate(subs):
                    wt += np.minimum(d[:, i], axes[p] - d[:, i])
                d = d[wt <= R]
            if not len(d):
                continue
            pp = np.zeros((len(d), w), dtype=np.int64)
            dd = np.zeros((len(d), w), dtype=np.int64)
            pp[:, :k] = subs
            dd[:, :k] = d
            P.append(pp)
            D.append(dd)
    return np.concatenate(P), np.concatenate(D)


def locality_key(pos, dlt, axes):
    """Unwrapped offset sum(delta * stride) of every pattern."""
    stride = np.cumprod([1] + [int(a) for a in axes[:-1]]).astype(np.int64)
    return (dlt * stride[pos]).sum(axis=1)


def wide_table(axes, R, problem, order=True):
    """Engine table: int32 (L, slots), (pos << 24) | delta per slot."""
    pos, dlt = enumerate_ball(axes, R, problem)
    if order:
        o = np.argsort(locality_key(pos, dlt, axes), kind="stable")
        pos, dlt = pos[o], dlt[o]
    if max(axes) >= 1 << 24:
        raise ValueError("axis too wide for the 24-bit delta field")
    tbl = np.where(dlt > 0, (pos << 24) | dlt, 0).astype(np.int32)
    return np.ascontiguousarray(tbl)


def v1_table(axes, R, problem, order=True):
    """Reference v1 packed table (uint64 per pattern)."""
    if max(axes) > 16 or len(axes) > 16:
        raise ValueError("the v1 table packs positions and deltas in "
                         "nibbles: at most 16 axes of size <= 16")
    pos, dlt = enumerate_ball(axes, R, problem)
    if pos.shape[1] > 8:
        raise ValueError("the v1 table holds at most 8 changed positions")
    if order:
        o = np.argsort(locality_key(pos, dlt, axes), kind="stable")
        pos, dlt = pos[o], dlt[o]
    byte = np.where(dlt > 0, (pos << 4) | dlt, 0).astype(np.uint64)
    out = np.zeros(len(pos), dtype=np.uint64)
    for k in range(pos.shape[1]):
        out |= byte[:, k] << np.uint64(8 * k)
    return out


def ball_size(axes, R, problem):
    return len(enumerate_ball(axes, R, problem)[0])
