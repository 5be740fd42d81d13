"""bench.py's host pieces: the clock record taken from nvidia-smi's CSV rows
during the timed region (median SM clock, max clock, throttle reasons seen
Active), the roofline denominators' fallback, and the workload description."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

ROW = "0, {sm}, 1965, 850.12, {act}, {hw}, Not Active, Not Active, {cap}"


def _rows(*specs):
    return "\n".join(ROW.format(sm=sm, act=act, hw=hw, cap=cap) for sm, act, hw, cap in specs)


def test_clock_record_median_and_reasons():
    text = _rows((1897, "0x4", "Not Active", "Active"),
                 (1905, "0x0", "Not Active", "Not Active"),
                 (1890, "0x4", "Not Active", "Active"))
    r = bench.ClockSampler.summarise(text)
    assert r == {"sm_mhz": 1897.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}


def test_clock_record_reports_a_hardware_slowdown():
    r = bench.ClockSampler.summarise(_rows((1200, "0x8", "Active", "Not Active")))
    assert r["reasons"] == ["hw_slowdown"] and r["sm_mhz"] == 1200.0


def test_clock_record_skips_rows_that_do_not_parse():
    text = "\n".join(["", "garbage", "0, [N/A], 1965, 1, x, Not Active, Not Active, Not Active, Not Active",
                      _rows((1800, "0x0", "Not Active", "Not Active"))])
    r = bench.ClockSampler.summarise(text)
    assert r["samples"] == 1 and r["sm_mhz"] == 1800.0 and r["reasons"] == []
    assert bench.ClockSampler.summarise("") == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                                                "samples": 0}


def test_unstarted_sampler_says_so():
    r = bench.ClockSampler(0).stop()
    assert r["samples"] == 0 and r["reasons"] == ["nvidia-smi unavailable"]


def test_peak_source_and_workload_description():
    hbm, source = bench.measured_peaks()
    assert source in ("measured", "fallback") and hbm > 1000.0
    if source == "fallback":
        assert hbm == 6650.0
    d = bench.config_dict(4096, "fast", {"extra": 1})
    assert d["grid"] == [4096, 4096] and d["arith_mode"] == "fast" and d["extra"] == 1
    assert "4096x4096" in d["workload"] and "model" not in d
    assert bench.BYTES_PER_ZU_RK2 == 5 * 4 * 8
