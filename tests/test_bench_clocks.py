"""The bench's clock record, taken on a fake NVML (no GPU): the sampler
polls while the timed region runs, reports the median SM clock, the maximum
clock and every clock-event reason seen (sw_power_cap kept, slowdowns named),
and makes read-only queries only."""
import threading
import time

import bench


class FakeNVML:
    NVML_CLOCK_SM = 0
    nvmlClocksEventReasonHwSlowdown = 0x8
    nvmlClocksEventReasonHwThermalSlowdown = 0x40
    nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nvmlClocksEventReasonSwPowerCap = 0x4

    def __init__(self, clocks, reasons):
        self.clocks, self.reasons, self.k = clocks, reasons, 0

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return self.reasons[min(self.k, len(self.reasons) - 1)]

    def nvmlDeviceGetClockInfo(self, h, kind):
        v = self.clocks[min(self.k, len(self.clocks) - 1)]
        self.k += 1
        return v

    def nvmlDeviceGetPowerUsage(self, h):
        return 650000


def run(nv, seconds=0.08):
    c = bench.ClockSampler(0)
    c.nv, c.h, c.max_mhz = nv, None, 1965
    c.done, c.first = threading.Event(), threading.Event()
    c.t = threading.Thread(target=c._poll, daemon=True)
    c.t.start()
    assert c.first.wait(2.0)
    time.sleep(seconds)
    return c.stop()


def test_median_and_power_cap():
    r = run(FakeNVML([1965, 1950, 1965, 1965], [0x4]))
    assert r["source"] == "NVML, 10 ms" and r["samples"] >= 3
    assert r["sm_mhz"] == 1965 and r["sm_max_mhz"] == 1965
    assert r["reasons"] == ["sw_power_cap"] and r["power_w_median"] == 650.0


def test_slowdowns_are_named():
    r = run(FakeNVML([1400], [0x0, 0x8 | 0x40]))
    assert r["reasons"] == ["hw_slowdown", "hw_thermal_slowdown"]
    assert r["sm_mhz"] == 1400
