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


def test_stratified_sample_covers_every_size():
    import bench
    counts = [5, 300, 12, 40, 41, 7, 250, 90, 8, 60]
    idx = bench.stratified_sample(counts, 5)
    assert len(idx) == len(set(idx)) == 5
    picked = sorted(counts[i] for i in idx)
    assert picked[0] <= 8 and picked[-1] >= 250   # both ends of the size range are in the sample
    assert sorted(bench.stratified_sample(counts, 100)) == list(range(10))


def test_cpu_baseline_rate_is_load_balanced():
    """Two scenes of very different cost on two cores: the rate is cores x scenes / sum of the per-scene step
    times (a balanced host), not the scene-steps of the slowest worker."""
    import argparse
    import bench
    from conftest import load_fixture
    small, big = load_fixture("boxes8"), load_fixture("c1_boxes64")
    args = argparse.Namespace(termination="merit", cpu_scenes=2, scheme="rigid_gauss_seidel", tolerance=1e-6,
                              ordering="serial", residual_interval=1, no_warm_start=True, max_iterations=None,
                              cpu_seconds=0.2, pre_roll=2)
    rate, info = bench.cpu_baseline([small, big], args, 1)
    t = info["seconds_per_step_p50_max"]
    assert info["cores"] == 1 and "2 of 2 scenes" in info["sample"]
    # one core: the mix of the two scenes runs at 2 / (t_small + t_big) scene-steps/s, and the median of two
    # per-scene times is their mean
    assert rate > 0 and abs(1.0 / rate - t[0]) <= 1e-9 / rate
    assert info["body_steps_per_s"] > rate
