"""bench.py's host-side helpers, without a GPU: the clock-sample parser,
the launch-form names, the traffic lookup and the peak fallback."""
import json
import os

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_clock_samples():
    text = ("0, 1965, 1965, 650.1, 0x0000000000000000, Not Active, "
            "Not Active, Not Active, Not Active\n"
            "0, 1950, 1965, 990.0, 0x0000000000000004, Not Active, "
            "Not Active, Not Active, Active\n"
            "garbage line\n"
            "0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, "
            "Not Active\n")
    c = bench.parse_clock_samples(text)
    assert c == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0,
                 "reasons": ["sw_power_cap"], "samples": 3}
    assert bench.parse_clock_samples("") is None
    hot = "0, 1500, 1965, 1000, 0x8, Active, Not Active, Not Active, Active"
    assert bench.parse_clock_samples(hot)["reasons"] == ["hw_slowdown",
                                                         "sw_power_cap"]


def test_form_names():
    assert bench.form_name(0) == "plain"
    assert bench.form_name(1 | 2 | 4 | 8) == "pipe+pack+in16+out16"
    assert bench.form_name(2 | 8 | 16) == "pack+out16+pair"


def test_traffic_covers_every_h2_grouping():
    """Each grouping the autotuner can choose for H2(26,3) has a capture
    for every launch (the planner gives the same groupings on the host)."""
    from coldcore_b200.gpu import plan_probe
    with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
        traffic = json.load(f)
    for budget, pipe in ((100, 1), (160, 1), (64, 1), (200, 1), (100, 2),
                         (100, 3), (200, 3), (160, 2), (200, 2)):
        for mode, key in (((0, 2), "(0,2)"), ((1, 1), "(1,1)"),
                          ((2, 1), "(2,1)")):
            for L in plan_probe("hamming", [2] * 26, 3, *mode,
                                budget_kb=budget, pipe=pipe):
                axes = f"{L['axis0']}..{L['axis0'] + L['axes'] - 1}"
                k = f"H2_26_3:{key}:{axes}"
                assert bench.ncu_traffic(k) == traffic[k] > 0, k


def test_peak_fallback_or_measured():
    peak, kind = bench.peaks()
    assert kind in ("measured", "fallback") and peak > 1000


def test_out_of_hbm_projection_is_in_seconds():
    """17.18 GB crossed in 310.9 ms is 55.3 GB/s; the reference's K_10(10,5)
    link traffic (240 GB) at that rate takes 4.34 s."""
    from harness.ooc_bench import K10_LINK_BYTES, link_projection_s
    assert K10_LINK_BYTES == 240 * 10 ** 9
    s = link_projection_s(17179869184, 310.907)
    assert abs(s - 4.343) < 0.01
