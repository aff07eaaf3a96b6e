"""bench.py's host-side pieces that need no GPU: the clock summary the JSON line carries."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def _sampler(samples):
    import bench
    c = bench.ClockSampler.__new__(bench.ClockSampler)   # no NVML, no thread: only the summary is tested
    c.samples = samples
    return c


def test_clock_summary_median_and_reasons():
    busy = ["0", "1965", "1965", "800.0", "0x0", "Not Active", "Not Active", "Not Active", "Not Active"]
    capped = ["0", "1800", "1965", "1000.0", "0x4", "Not Active", "Not Active", "Not Active", "Active"]
    s = _sampler([busy, busy, capped]).summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"]
    hot = ["0", "1200", "1965", "900.0", "0x40", "Not Active", "Active", "Not Active", "Not Active"]
    assert _sampler([hot]).summary()["reasons"] == ["hw_thermal_slowdown"]


def test_clock_summary_without_samples():
    assert _sampler([]).summary()["reasons"] == ["unsampled"]
