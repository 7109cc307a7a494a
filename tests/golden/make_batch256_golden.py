#!/usr/bin/env python3
"""Golden digests of the 256-cell batched campaign workload.

For every cell of ``coldcore_b200.workloads.batch_cells(256, seed=7)`` (the
configuration the bench's batched leg times), the C restatement of the
reference's CPU axis DP (``oracle/cport``, pinned to the numpy oracle by
``tests/test_cport.py``) computes cnt from the cell's code, the gain map
and the loss map; this script records the first 16 hex digits of the
SHA-256 of each field's bytes (cnt as uint16, maps as int32, little-endian)
and the three scalars (deficit at mu = 1, gain maximum, loss maximum):

    python tests/golden/make_batch256_golden.py     # about a minute

Output: ``batch256_golden.json`` (committed; the GPU test compares the
batched engine's fields with these digests).
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from coldcore_b200.workloads import batch_cells   # noqa: E402
from oracle.cport import CPortCell                 # noqa: E402


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def main():
    out = []
    for i, (p, a, R, code) in enumerate(batch_cells(256, seed=7)):
        c = CPortCell(list(a), R, p)
        c.recount(code)
        row = {"cell": i, "problem": p, "axes": list(a), "R": R,
               "M": int(len(code)), "cnt": digest(c.cnt.astype("<u2")),
               "deficit": int((c.cnt == 0).sum())}
        c.gain_map()
        row["gain"], row["gain_max"] = digest(c.map.astype("<i4")), \
            int(c.map.max())
        c.loss_map()
        row["loss"], row["loss_max"] = digest(c.map.astype("<i4")), \
            int(c.map.max())
        out.append(row)
    with open(os.path.join(HERE, "batch256_golden.json"), "w") as f:
        f.write("[\n" + ",\n".join(json.dumps(r) for r in out) + "\n]\n")


if __name__ == "__main__":
    main()
