"""bench.py's clock record: the samples taken inside the timed region are
the ones summarised, and a region shorter than the sampling interval falls
back to the nearest sample (host logic only, with synthetic samples)."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402


def _row(mhz, power_cap="Not Active", thermal="Not Active"):
    return [str(mhz), "1965", "700.0", "Not Active", "Not Active", thermal, power_cap]


def test_clock_summary_keeps_the_timed_region():
    c = bench.ClockSampler(0)
    c.rows = [(0.00, _row(1200, thermal="Active")), (0.05, _row(1965)), (0.10, _row(1950, "Active")),
              (0.15, _row(1965)), (0.20, _row(900))]
    c.mark(0.04, 0.16)
    s = c.summary()
    assert s["samples"] == 3 and s["samples_from"] == "timed region"
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]  # the thermal sample lies outside


def test_clock_summary_nearest_sample_when_none_inside():
    c = bench.ClockSampler(0)
    c.rows = [(0.0, _row(1800)), (0.3, _row(1965))]
    c.mark(0.20, 0.26)
    s = c.summary()
    assert s["samples"] == 1 and s["sm_mhz"] == 1965.0 and s["samples_from"].startswith("nearest")


def test_clock_summary_unsampled():
    assert bench.ClockSampler(0).summary()["reasons"] == ["unsampled"]
