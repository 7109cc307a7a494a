"""Byte models of the covering transforms.

``model_bytes`` is the one-axis-per-pass traffic of a whole-space
transform — the byte model the reference's own transform benchmark uses as
its bandwidth yardstick (coldcore ``scripts/bench_transform.py:30-38``),
refined with zero-layer skipping: pass j reads min(j,R)+1 int32 planes
(pass 0 reads the 2-byte cnt for gain / loss, the 4-byte A0 for a
recount) and writes min(j+1,R) planes (plus layer 0 on pass 0); the last
pass writes the 4-byte map or the 2-byte cnt; a recount also fills A0.
Window families (torus / grid) move one plane per pass.  Dividing it by a
transform's time gives the same "transform GB/s" for every
implementation, so ratios of it are speed ratios.
"""


def model_bytes(axes, R, problem, mode):
    """Bytes per transform; mode 'recount' (code -> cnt) or 'gain' /
    'loss' (cnt predicate -> map)."""
    n = len(axes)
    size = 1
    for a in axes:
        size *= int(a)
    recount = mode == "recount"
    if problem in ("torus_linf", "grid_linf"):
        per = 0
        for j in range(n):
            rd = (4 if recount else 2) if j == 0 else 4
            wr = (2 if recount else 4) if j == n - 1 else 4
            per += rd + wr
        if recount:
            per += 4
        return per * size
    per = 0
    for j in range(n):
        lin = min(j, R) + 1
        lout = min(j + 1, R) + 1
        rd = (4 if recount else 2) if j == 0 else 4 * lin
        if j == n - 1:
            wr = 2 if recount else 4
        else:
            wr = 4 * (lout - 1) + (4 if j == 0 else 0)
        per += rd + wr
    if recount:
        per += 4
    return per * size
