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


def test_reference_arm_loads_only_the_oracle():
    """bench.py --impl reference builds its mesh, operator and particles with
    the oracle alone: the process maps no library of the product, and its
    JSON line carries the same config keys as the product arm."""
    import json
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys, os; sys.argv = ['bench.py', '--impl', 'reference', '--config', 'cfg1', "
            "'--cpu-sample', '2000', '--steps', '1']; sys.path.insert(0, %r); import bench; bench.main(); "
            "print('SO', sorted({l.split()[-1] for l in open('/proc/self/maps') "
            "if l.rstrip().endswith('.so') and %r in l}))" % (root, root))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    line = json.loads([l for l in lines if l.startswith("{")][0])
    so = __import__("ast").literal_eval(lines[-1][3:])
    assert so == [os.path.join(root, "oracle", "liboracle.so")], so
    assert line["impl"] == "reference" and line["dtype"] == "f64"
    assert set(line["config"]) >= {"workload", "cells", "particles", "precision", "pcg_tol", "mcc"}
    assert line["config"]["particles"] > 300000 and line["value"] > 0
