"""bench.py's host logic on the CPU: the clock record taken during the timed region (median SM
clock, maximum, throttle reasons as nvidia-smi prints them), the roofline denominator read from
the measured peaks, and the whole-job rate.  No GPU is involved."""
import json

import bench


def _sampler(rows):
    s = bench.ClockSampler()
    s.samples = [[x.strip() for x in r.split(",")] for r in rows]
    return s


def test_clock_summary_median_max_and_reasons():
    s = _sampler(["1965, 1965, Not Active, Not Active, Not Active, Not Active",
                  "1800, 1965, Not Active, Not Active, Not Active, Active",
                  "1900, 1965, Not Active, Not Active, Not Active, Not Active"])
    out = s.summary()
    assert out["sm_mhz"] == 1900.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"] and out["samples"] == 3


def test_clock_summary_reports_slowdowns_and_skips_unreadable_values():
    s = _sampler(["[N/A], 1965, Active, Not Active, Not Active, Not Active",
                  "1200, 1965, Not Active, Active, Active, Not Active"])
    out = s.summary()
    assert out["sm_mhz"] == 1200.0
    assert out["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]


def test_clock_summary_without_samples():
    assert bench.ClockSampler().summary()["reasons"] == ["unsampled"]


def test_peaks_reads_the_measured_copy_bandwidth(tmp_path, monkeypatch):
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6545.0}))
    monkeypatch.setattr(bench, "REPO", str(tmp_path))
    assert bench.peaks() == (6545.0, "measured")
    monkeypatch.setattr(bench, "REPO", str(tmp_path / "absent"))
    assert bench.peaks() == (6650.0, "fallback")


def test_whole_job_rate_counts_every_rank():
    assert bench.whole_job_rate(1, 64, 16.0) == 4000.0
    assert bench.whole_job_rate(8, 64, 16.0) == 32000.0
