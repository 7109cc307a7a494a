"""CPU oracle for the coldcore covering transforms — TEST INFRASTRUCTURE ONLY.

Nothing in ``coldcore_b200`` imports this package.  It is the checker: the
``tests/`` suite, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` are its only callers.

Contents
--------
``dp_oracle``   numpy restatement of the reference's axis-DP backend
                (coldcore ``src/coldcore/dp.py``) with int64 digits, so the
                ball walks stay correct on axes wider than 255 (the reference
                returns uint8 digits from ``ProductSpace.index_word``,
                ``src/coldcore/space.py:34-36``).
``brute``       O(|X|^2) restatement of the reference's brute-force backends
                (``src/coldcore/reference/*.py``), tiny spaces only.
``cport``       the same axis DP as plain C (OpenMP over fibres), the timed
                CPU baseline of ``bench.py``.

Pinning: ``tests/golden/make_golden.py`` imported the reference's own numpy
backends from the reference checkout and wrote the committed fixtures under
``tests/golden/``; ``tests/test_oracle_golden.py`` checks this oracle against
every one of them.
"""
