"""The benchmark's clock record on the host: NVML polled during the timed
region (here a fake NVML module: reading clocks needs no GPU settings), and
the fallback when NVML cannot start."""
import itertools
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


class FakeNvml:
    NVML_CLOCK_SM = 1

    def __init__(self, clocks, reasons, fail_init=False):
        self.clocks = itertools.cycle(clocks)
        self.reasons = itertools.cycle(reasons)
        self.fail_init = fail_init
        self.shutdown = False

    def nvmlInit(self):
        if self.fail_init:
            raise RuntimeError("NVML library not found")

    def nvmlShutdown(self):
        self.shutdown = True

    def nvmlDeviceGetHandleByPciBusId(self, bus_id):
        return ("pci", bus_id)

    def nvmlDeviceGetHandleByIndex(self, i):
        return ("index", i)

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        assert kind == self.NVML_CLOCK_SM
        return 1965

    def nvmlDeviceGetClockInfo(self, h, kind):
        assert kind == self.NVML_CLOCK_SM
        return next(self.clocks)

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return next(self.reasons)


def test_nvml_samples_inside_the_timed_region():
    nv = FakeNvml([1965, 1965, 1950], [0x0, 0x4, 0x1])  # 0x4: sw power cap, 0x1: idle (not reported)
    c = bench.ClockSampler(0, nvml=nv)
    c.start()
    time.sleep(0.02)
    c.mark_start()
    time.sleep(0.05)
    c.mark_end()
    time.sleep(0.02)
    r = c.stop()
    assert nv.shutdown
    assert r["source"] == "NVML every 2 ms, timed region"
    assert r["sm_max_mhz"] == 1965.0
    assert r["sm_mhz"] in (1950.0, 1965.0)
    assert r["reasons"] == ["sw_power_cap"]
    # only the samples inside the window count: fewer than all that were taken
    assert 3 <= r["samples"] < len(c.samples)
    assert r["samples"] == sum(c.t0 <= t <= c.t1 for t, _, _ in c.samples)


def test_nvml_throttle_bits_map_to_reported_reasons():
    nv = FakeNvml([1200], [0x8 | 0x40 | 0x20])
    c = bench.ClockSampler(0, nvml=nv)
    c.start()
    c.mark_start()
    time.sleep(0.02)
    c.mark_end()
    r = c.stop()
    assert r["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]
    assert r["sm_mhz"] == 1200.0


def test_without_marks_the_whole_run_counts():
    c = bench.ClockSampler(0, nvml=FakeNvml([1965], [0]))
    c.start()
    time.sleep(0.01)
    r = c.stop()
    assert r["source"] == "NVML every 2 ms, whole run" and r["samples"] >= 1


def test_falls_back_when_nvml_cannot_start(monkeypatch):
    """NVML unavailable: the nvidia-smi sampler runs instead; with no
    nvidia-smi either (this host has none), the record is None."""
    started = []
    monkeypatch.setattr(bench.ClockSampler, "_start_smi", lambda self: started.append(True))
    c = bench.ClockSampler(0, nvml=FakeNvml([1965], [0], fail_init=True))
    c.start()
    assert started == [True] and c.thread is None
    assert c.stop() is None
