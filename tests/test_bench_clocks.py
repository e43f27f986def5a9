"""Clock sampling of bench.py on CPU, against a fake NVML module: the samples taken while the
timed region runs, the clock-event (throttle) reasons decoded from the NVML bit mask, and the
fallback when NVML cannot be used.  Only read-only queries exist in the fake: the sampler sets
nothing."""
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


class FakeNVML:
    NVML_CLOCK_SM = 1
    nvmlClocksEventReasonSwPowerCap = 0x4
    nvmlClocksEventReasonHwSlowdown = 0x8
    nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nvmlClocksEventReasonHwThermalSlowdown = 0x40

    def __init__(self, mask=0, clocks=(1965, 1950, 1965), fail=False):
        self.mask, self.clocks, self.fail = mask, clocks, fail
        self.calls = 0
        self.shut = False

    def nvmlInit(self):
        if self.fail:
            raise RuntimeError("NVML unavailable")

    def nvmlShutdown(self):
        self.shut = True

    def nvmlDeviceGetHandleByIndex(self, i):
        return ("gpu", i)

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        assert kind == self.NVML_CLOCK_SM
        return 1965

    def nvmlDeviceGetClockInfo(self, h, kind):
        self.calls += 1
        return self.clocks[self.calls % len(self.clocks)]

    def nvmlDeviceGetPowerUsage(self, h):
        return 612_000          # mW

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return self.mask


def test_nvml_samples_during_the_region_and_decodes_reasons():
    nv = FakeNVML(mask=0x4 | 0x1)     # power cap and GPU idle (not reported)
    c = bench.Clocks(0, nvml=nv)
    c.start()
    time.sleep(0.25)
    r = c.stop()
    assert r["source"] == "nvml" and nv.shut
    assert r["samples"] >= 5           # one every 20 ms
    assert r["sm_max_mhz"] == 1965 and r["power_w_max"] == 612.0
    assert 1950 <= r["sm_mhz"] <= 1965
    assert r["reasons"] == ["sw_power_cap"]


def test_nvml_reports_every_slowdown_reason():
    nv = FakeNVML(mask=0x8 | 0x20 | 0x40)
    c = bench.Clocks(0, nvml=nv)
    c.start()
    time.sleep(0.05)
    r = c.stop()
    assert r["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]


def test_without_nvml_falls_back_without_raising():
    c = bench.Clocks(0, nvml=FakeNVML(fail=True))
    c.start()
    r = c.stop()
    # nvidia-smi (absent here: no record) or its samples; never an exception
    assert r is None or r["source"] == "nvidia-smi"
