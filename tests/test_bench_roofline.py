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
    variants = {"carry_chain_probe": 12.0, "independent_mad_probe": 18.0}
    conv = (1 << 20) * 176 * 264 / 4e-3 / 1e12
    issued = (1 << 20) * 13 * bench.ISSUED_IMAD_PER_RECORD["accum_g1"] / 4e-3 / 1e12
    # the default headline is the fixed algorithmic work, issued beside it
    r0 = bench.roofline_of("accum_g1", (4.0, 1, float(1 << 20)), 12.0, None, 13, variants)
    assert r0["work"] == "convention" and abs(r0["frac"] - conv / 12.0) < 1e-12
    assert abs(r0["issued"]["frac"] - issued / 12.0) < 1e-12
    r = bench.roofline_of("accum_g1", (4.0, 1, float(1 << 20)), 12.0, None, 13, variants,
                          headline="issued")
    assert r["work"] == "issued"
    assert abs(r["achieved"] - issued) < 1e-9 and abs(r["frac"] - issued / 12.0) < 1e-12
    assert abs(r["convention"]["achieved"] - conv) < 1e-9
    assert abs(r["issued"]["achieved"] - issued) < 1e-9
    assert r["frac"] < r["convention"]["frac"]
    assert abs(r["peak_variants"]["independent_mad_probe"]["frac"] - issued / 18.0) < 1e-12
    # without the window count the convention is the headline
    r2 = bench.roofline_of("accum_g1", (4.0, 1, float(1 << 20)), 12.0, None)
    assert r2["work"] == "convention" and abs(r2["frac"] - conv / 12.0) < 1e-12
    assert bench.roofline_of("accum_g2", (0.0, 0, 0.0), 12.0, None, 13) is None


def test_parity_report_flags_any_difference():
    mine = {"proof_2^20": "aa", "g1_msm": {"2^18": "x", "2^20": "y"}, "ntt": {"2^16": "d"}}
    ref = {"proof_2^20": "aa", "primitives": {"g1_msm": {"2^18": "x", "2^20": "y"},
                                              "ntt": {"2^16": "d"}}}
    r = bench.parity_report(mine, ref, "test")
    assert r["all_equal"] and r["proof_2^20"] and r["g1_msm"]["2^20"]
    ref["primitives"]["g1_msm"]["2^20"] = "z"
    r = bench.parity_report(mine, ref, "test")
    assert not r["all_equal"] and r["g1_msm"]["2^20"] is False
    # items the reference did not run are reported as unchecked, not equal
    r = bench.parity_report({"proof_2^22": "bb"}, {"primitives": {}}, "test")
    assert r["proof_2^22"] is None and r["all_equal"]
    assert bench.parity_report(mine, None, "absent") == {"checked": False, "source": "absent"}
