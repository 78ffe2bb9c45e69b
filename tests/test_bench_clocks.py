"""bench.py's clock sampler on the CPU, against a fake NVML and a fake nvidia-smi stream: the
median SM clock, the maximum power and the clock-event reasons of the samples.  (It only reads
the GPU's state.)"""
import sys
import threading
import time

from conftest import ROOT

sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


class FakeNvml:
    NVML_CLOCK_SM = 1

    def __init__(self):
        self.calls = 0

    def nvmlDeviceGetMaxClockInfo(self, handle, kind):
        return 1965

    def nvmlDeviceGetClockInfo(self, handle, kind):
        self.calls += 1
        return 1400 if self.calls % 2 else 1500

    def nvmlDeviceGetPowerUsage(self, handle):
        return 990_000 if self.calls == 3 else 700_000  # milliwatts

    def nvmlDeviceGetCurrentClocksEventReasons(self, handle):
        return 0x4 | (0x40 if self.calls == 2 else 0)  # power cap; one thermal slowdown sample


def test_nvml_sampler_reports_median_clock_and_every_reason():
    s = bench.ClockSampler(0, "GPU-fake")
    fake = FakeNvml()
    s._nvml_handle = lambda: (fake, None)
    s.start()
    time.sleep(0.15)
    out = s.stop()
    assert out["source"].startswith("NVML") and out["samples"] >= 5
    assert out["sm_max_mhz"] == 1965.0
    assert 1400.0 <= out["sm_mhz"] <= 1500.0
    assert out["power_w_max"] == 990.0
    assert out["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]


def test_nvidia_smi_fallback_parses_the_query_lines():
    s = bench.ClockSampler(0)
    s.nvml = None

    class Done:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            return 0

    s.proc = Done()
    s.thread = threading.Thread(target=lambda: None)
    s.thread.start()
    s.lines = ["0, 1410, 1965, 995.1, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1420, 1965, 998.0, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1965, 1965, 300.0, 0x0, Not Active, Not Active, Not Active, Not Active",
               "garbage"]
    out = s.stop()
    assert out["samples"] == 3 and out["sm_mhz"] == 1420.0 and out["sm_max_mhz"] == 1965.0
    assert out["power_w_max"] == 998.0 and out["reasons"] == ["sw_power_cap"]
    assert out["source"].startswith("nvidia-smi")


def test_no_sampler_available():
    s = bench.ClockSampler(0)
    s.nvml = None
    s.proc = None
    assert s.stop()["sm_mhz"] is None
