"""The mixed-radix product space X = Z_{a_0} x ... x Z_{a_(n-1)}.

A word (d_0, ..., d_(n-1)) has the index x = sum_j d_j * s_j with the
little-endian strides s_j = a_0 * ... * a_(j-1); that numbering is the one
coldcore's cells, codes and cover files use (``src/coldcore/space.py:10-45``
defines the same numbering).  Digits here are int64 throughout, so axes
wider than 255 round-trip (coldcore's ``index_word`` returns uint8 digits).

The conversions are single vectorised expressions over the stride vector:
an index's digit j is ``(x // s_j) mod a_j``.
"""
import numpy as np


class ProductSpace:
    """``ProductSpace(q, n)`` for the homogeneous space Z_q^n, or
    ``ProductSpace(axes)`` for a mixed radix; exposes ``axes``, ``n``,
    ``q`` (None when mixed), ``size`` and the strides ``pow_q``."""

    def __init__(self, q_or_axes, n=None):
        radix = (np.full(int(n), int(q_or_axes), dtype=np.int64)
                 if n is not None else
                 np.array([int(a) for a in q_or_axes], dtype=np.int64))
        if radix.ndim != 1 or np.any(radix < 1):
            raise ValueError(f"bad axes {q_or_axes!r}")
        stride = np.ones(len(radix), dtype=np.int64)
        np.cumprod(radix[:-1], out=stride[1:])
        self._radix = radix
        self.pow_q = stride
        self.axes = radix.tolist()
        self.n = len(radix)
        self.size = int(np.prod(radix, dtype=np.int64))
        self.q = int(radix[0]) if self.n and np.all(radix == radix[0]) \
            else None

    def word_index(self, words):
        """(k, n) digit array -> int64 indices."""
        return np.asarray(words, dtype=np.int64) @ self.pow_q

    def index_word(self, idx):
        """int64 indices -> (k, n) int64 digit array."""
        x = np.asarray(idx, dtype=np.int64).reshape(-1, 1)
        return (x // self.pow_q) % self._radix

    def all_words(self):
        return self.index_word(np.arange(self.size, dtype=np.int64))
