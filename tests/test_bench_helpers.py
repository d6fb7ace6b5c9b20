"""Host-side helpers of bench.py that its JSON line depends on: the clock
summary (throttle reasons that reject a run) and the profile values read
from the committed summaries."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_clock_summary_collects_reasons_and_median():
    c = bench.ClockSampler(0)
    c.source = "test"
    c.rows = [(1965.0, 1965.0, set()), (1900.0, 1965.0, {"sw_power_cap"}), (1965.0, 1965.0, {"hw_slowdown"})]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_min_mhz"] == 1900.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"] and s["samples"] == 3


def test_clock_summary_without_samples_says_so():
    assert bench.ClockSampler(0).summary()["reasons"] == ["unsampled"]


def test_profile_values_come_from_committed_summaries():
    traffic = bench._profile_value("exact2nn_u8_pair_10000x1M.md", "traffic_bytes_per_launch")
    peak = bench._profile_value("tcgen05_int8_peak.md", "peak_int8_tops")
    assert traffic and traffic > 1e9
    assert peak and 4000 < peak < 5000
    assert bench._profile_value("no_such_file.md", "x") is None
