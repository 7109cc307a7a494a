"""Measurement harnesses that drive the engine from outside the package:
``profile_cell`` (one cell's transforms for a profiler capture),
``incidence_bench`` (the explicit-incidence field timing) and
``lns_study`` (the multi-seed learned-against-plain LNS study).
``bench.py`` imports the last two for its secondary legs."""
