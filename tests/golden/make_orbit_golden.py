"""Generate ``orbit_golden.npz``: the reference's own permutation groups
and design quotients (coldcore ``src/coldcore/problems/perm_groups.py``,
``design_orbits.py``) on seeded cases.

Needs the reference source tree on the path (default
``/root/reference/src``, override with ``COLDCORE_REF_SRC``):

    python tests/golden/make_orbit_golden.py

Records, per group spec: its order; per (v, r, spec): the r-subset orbit
labels; per (v, k, t, spec): the block and t-subset orbit sizes and
representatives and the quotient CSR with and without short orbits.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.environ.get("COLDCORE_REF_SRC", "/root/reference/src"))

from coldcore.problems.design_orbits import DesignOrbits  # noqa: E402
from coldcore.problems.perm_groups import parse_design_group  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
GROUPS = [(7, "cyclic"), (8, "cyclic-1"), (9, "cyclic-2"), (7, "dihedral"),
          (9, "prod:3x3"), (12, "prod:3x4"), (7, "affine"), (13, "affine:3"),
          (13, "mult:3"), (6, "gens=(0 1 2)(3 4);(5 0)"),
          (7, "cyclic+dihedral"), (5, "trivial")]
SUBSETS = [(7, 3, "cyclic"), (9, 3, "prod:3x3"), (8, 4, "dihedral"),
           (7, 2, "affine"), (10, 4, "cyclic-1")]
QUOTIENTS = [(7, 3, 2, "cyclic"), (9, 3, 2, "prod:3x3"), (8, 4, 2, "dihedral"),
             (9, 4, 3, "cyclic-1"), (13, 4, 2, "cyclic"), (11, 5, 3, "affine")]


def main():
    out = {}
    for v, spec in GROUPS:
        out[f"order/{v}/{spec}"] = np.int64(parse_design_group(v, spec).order())
    for v, r, spec in SUBSETS:
        part = parse_design_group(v, spec).subset_orbits(r)
        out[f"subsets/{v}/{r}/{spec}"] = part.labels
    for v, k, t, spec in QUOTIENTS:
        orb = DesignOrbits(v, k, t, spec)
        p = f"quotient/{v}/{k}/{t}/{spec}/"
        out[p + "block_sizes"] = orb.block_part.sizes
        out[p + "block_reps"] = orb.block_part.reps
        out[p + "univ_sizes"] = orb.univ_part.sizes
        out[p + "univ_reps"] = orb.univ_part.reps
        for short in (False, True):
            cand, indptr, indices, w, uw = orb.quotient_csr(short)
            q = p + ("short/" if short else "full/")
            out[q + "cand"] = cand
            out[q + "indptr"] = indptr
            out[q + "indices"] = indices
            out[q + "w"] = w
            out[q + "uw"] = uw
        print(orb.summary(), flush=True)
    path = os.path.join(HERE, "orbit_golden.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
