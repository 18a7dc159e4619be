"""Host logic of the bench line: the clock record (throttle reasons from
NVML's clock-event bit mask, the median SM clock, the nvidia-smi CSV
fallback; a fake NVML stands in for the GPU) and the count of our kernels
per step."""
import os
import sys
import types

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_nvml_samples_give_median_clock_and_active_reasons():
    c = bench.ClockSampler(0)
    c.max_mhz = 1965.0
    # sw_power_cap (0x4) in one sample, hw_thermal_slowdown (0x40) in another,
    # an unrelated bit (0x1, GPU idle) ignored
    c.samples = [(1965.0, 0x0), (1950.0, 0x4), (1900.0, 0x40 | 0x1)]
    s = c.summary()
    assert s["sm_mhz"] == 1950.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert s["source"] == "nvml"


def test_sampling_through_a_fake_nvml():
    fake = types.SimpleNamespace(NVML_CLOCK_SM=0)
    ticks = iter([1965, 1965, 1800, 1965] + [1965] * 10000)
    fake.nvmlDeviceGetClockInfo = lambda h, kind: next(ticks)
    fake.nvmlDeviceGetCurrentClocksEventReasons = lambda h: 0x8 if h == "slow" else 0x0
    c = bench.ClockSampler(0)
    c.nv, c.h = fake, "slow"
    c._sample()
    c._sample()
    s = c.summary()
    assert s["samples"] == 2 and s["reasons"] == ["hw_slowdown"]


def test_nvidia_smi_lines_are_the_fallback():
    c = bench.ClockSampler(0)
    c.lines = ["1965, 1965, 700.5, Not Active, Not Active, Not Active, Active",
               "1950, 1965, 710.0, Not Active, Not Active, Not Active, Not Active",
               "garbage"]
    s = c.summary()
    assert s["source"] == "nvidia-smi" and s["samples"] == 2
    assert s["sm_mhz"] == 1957.5 and s["sm_max_mhz"] == 1965.0 and s["reasons"] == ["sw_power_cap"]


def test_bc7_kernel_count_matches_the_pipeline():
    from block_compression_b200.settings import BC7Settings
    # alpha_basic: prep, the searches of mode 0, modes 1+3 (one launch) and
    # mode 7 (mode 2 skipped), the refines of modes 0, 1, 3 and 7, three
    # mode-4/5 launches, mode 6, select -- the 13 BC7 kernels of the
    # benchmark's launch list
    assert bench.bc7_kernel_count(BC7Settings.alpha_basic()) == 13
    # opaque_basic: no mode 7 candidates
    assert bench.bc7_kernel_count(BC7Settings.opaque_basic()) == 11
    # opaque_slow: mode 2 searched too
    assert bench.bc7_kernel_count(BC7Settings.opaque_slow()) == 13
