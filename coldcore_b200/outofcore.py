"""Streaming plans for cells whose layer planes exceed device memory.

A transform is a product of per-axis recurrences, so the axes can be
applied in two phases, each of which touches the planes in pieces that fit
the device:

* phase 1, **slabs**: the low axes 0..s-1 act inside contiguous slabs of
  ``h`` whole rows of ``P_low = a_0 ... a_{s-1}`` words: copy a slab of
  every live layer in, run the low axes on it, copy it back;
* phase 2, **columns**: the high axes s..n-1 act inside column blocks: the
  words ``[x0, x0 + w)`` of every one of the ``P_high = a_s ... a_{n-1}``
  rows, a pitched 2-D region (pitch ``P_low`` words) of each layer plane.

The host copy of the planes is read and written once per phase, so the
host-device traffic is ``2 phases x 2 directions x layers x |X|`` words.
The reference streams its layers from the GH200's coherent host memory
instead (src/plugins/covering/dctcore_core.cuh:86-119); a B200 host has no
coherent C2C, hence explicit copies.  This module plans the pieces; the
plan's geometry is what a device executor copies and launches on.
"""
from math import prod


def plan_stream(axes, nlayers, bytes_per_word, budget_bytes, buffers=2,
                min_width=32):
    """The split and the piece sizes for streaming a cell of ``axes``.

    ``budget_bytes`` is the device memory given to the pieces, ``buffers``
    the pieces resident at once (2: one computing while the next copies).
    Phase 1 takes the largest low block ``P_low`` whose slab of one row
    fits; phase 2 then needs columns of at least ``min_width`` words (or
    the whole row when it is shorter).  Returns a dict with ``split``
    (s), ``p_low``, ``p_high``, ``slab_rows`` (h), ``n_slabs``,
    ``col_width`` (w), ``n_cols`` and ``host_words`` (host-device words
    moved by both phases); raises ``ValueError`` when no two-phase split
    fits the budget."""
    axes = [int(a) for a in axes]
    if not axes or min(axes) < 1:
        raise ValueError("axes must be positive")
    if nlayers < 1 or bytes_per_word < 1 or buffers < 1:
        raise ValueError("nlayers, bytes_per_word and buffers must be >= 1")
    cap = int(budget_bytes) // (int(nlayers) * int(bytes_per_word)
                                * int(buffers))        # words per piece
    if cap < 1:
        raise ValueError("budget below one word of every layer")
    n = len(axes)
    size = prod(axes)
    best = None
    for s in range(1, n):
        p_low = prod(axes[:s])
        p_high = size // p_low
        if p_low > cap:
            break
        width_cap = cap // p_high
        need = min(min_width, p_low)
        if width_cap >= need:
            best = (s, p_low, p_high, width_cap)
    if best is None:
        raise ValueError(f"no two-phase split of {axes} fits {budget_bytes} "
                         f"bytes ({nlayers} layers x {bytes_per_word} B)")
    s, p_low, p_high, width_cap = best
    h = max(1, min(p_high, cap // p_low))
    w = min(p_low, width_cap)
    if w >= min_width:
        w -= w % min_width              # whole 128-byte lines at 4 B/word
    return {"split": s, "p_low": p_low, "p_high": p_high,
            "slab_rows": h, "n_slabs": -(-p_high // h),
            "col_width": w, "n_cols": -(-p_low // w),
            "host_words": 4 * nlayers * size}


def slabs(plan):
    """Phase-1 pieces: (first word, words) of each contiguous slab."""
    step = plan["slab_rows"] * plan["p_low"]
    total = plan["p_low"] * plan["p_high"]
    return [(x, min(step, total - x)) for x in range(0, total, step)]


def columns(plan):
    """Phase-2 pieces: (first low word, width) of each column block; the
    block is that range of every one of the ``p_high`` rows."""
    w, p_low = plan["col_width"], plan["p_low"]
    return [(x, min(w, p_low - x)) for x in range(0, p_low, w)]
