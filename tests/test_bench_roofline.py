"""bench.py's roofline arithmetic on CPU: the conventional work count and
the issued-work count of the fixed-base accumulation."""
import os
import sys
import types

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_table_windows_from_flag_tuning_and_default():
    a = types.SimpleNamespace(table_c="17,0", log_domain=20)
    tuned = ["msm 1 20 0 20 0 128 16 16", "table 1 20 0 20", "table 2 20 0 19"]
    assert bench.table_windows(a, tuned, 1) == 254 // 17 + 1  # the flag wins
    assert bench.table_windows(a, tuned, 2) == 254 // 19 + 1  # tuned entry
    assert bench.table_windows(a, "defaults", 2) == 254 // 20 + 1  # default for 2^20


def test_issued_fraction_counts_records_and_issued_ops():
    # one G1 launch of 2^20 points in 4 ms, 13 records per point
    r = bench.roofline_of("accum_g1", (4.0, 1, float(1 << 20)), 12.0, None, 13)
    conv = (1 << 20) * 176 * 264 / 4e-3 / 1e12
    assert abs(r["achieved"] - conv) < 1e-9 and abs(r["frac"] - conv / 12.0) < 1e-12
    issued = (1 << 20) * 13 * bench.ISSUED_IMAD_PER_RECORD["accum_g1"] / 4e-3 / 1e12
    assert abs(r["issued"]["achieved"] - issued) < 1e-9
    assert r["issued"]["frac"] < r["frac"]
    assert bench.roofline_of("accum_g2", (0.0, 0, 0.0), 12.0, None, 13) is None
