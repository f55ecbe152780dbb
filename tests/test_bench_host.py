"""Host-side parts of bench.py: the clock sampler's NVML path (against a fake
NVML library) and its fallback."""

from __future__ import annotations

import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402


class FakeNVML:
    NVML_CLOCK_SM = 1

    def __init__(self, reasons=0x4, fail_init=False):
        self.reasons, self.fail_init = reasons, fail_init
        self.bus_ids, self.shutdowns = [], 0

    def nvmlInit(self):
        if self.fail_init:
            raise RuntimeError("no driver")

    def nvmlShutdown(self):
        self.shutdowns += 1

    def nvmlDeviceGetHandleByPciBusId(self, bus_id):
        self.bus_ids.append(bus_id)
        return "gpu"

    def nvmlDeviceGetHandleByIndex(self, index):
        return "gpu"

    def nvmlDeviceGetMaxClockInfo(self, h, clock):
        return 1965

    def nvmlDeviceGetClockInfo(self, h, clock):
        return 1890

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return self.reasons


def test_nvml_sampling_and_reasons():
    nv = FakeNVML(reasons=0x4 | 0x40)
    with bench.ClockSampler(0, "00000000:1B:00.0", nvml=nv, period_s=0.001) as clk:
        time.sleep(0.05)
    s = clk.summary()
    assert s["source"] == "nvml" and s["samples"] >= 5
    assert s["sm_mhz"] == 1890 and s["sm_max_mhz"] == 1965
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert nv.bus_ids == ["00000000:1B:00.0"] and nv.shutdowns == 1


def test_no_reason_active():
    with bench.ClockSampler(0, nvml=FakeNVML(reasons=0), period_s=0.001) as clk:
        time.sleep(0.02)
    assert clk.summary()["reasons"] == []


class OlderNVML(FakeNVML):
    """A driver library without the clock-event name (only the throttle one)."""

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        raise RuntimeError("function not found")

    def nvmlDeviceGetCurrentClocksThrottleReasons(self, h):
        return 0x8


def test_throttle_reasons_name_of_older_drivers():
    with bench.ClockSampler(0, nvml=OlderNVML(), period_s=0.001) as clk:
        time.sleep(0.02)
    s = clk.summary()
    assert s["source"] == "nvml" and s["reasons"] == ["hw_slowdown"]


def test_fallback_when_nvml_does_not_load():
    with bench.ClockSampler(0, nvml=FakeNVML(fail_init=True)) as clk:
        time.sleep(0.01)
    assert clk.source == "nvidia-smi"
    s = clk.summary()
    if not clk.samples:  # no nvidia-smi on this host
        assert s["reasons"] == ["nvidia-smi unavailable"]


def test_stage_names_cover_the_header_stages():
    import re

    text = open(os.path.join(os.path.dirname(bench.__file__), "include", "gsht.h")).read()
    stages = dict((k, int(v)) for k, v in re.findall(r"\b(GSHT_STAGE_[A-Z_]+)\s*=\s*(\d+)", text))
    assert len(bench.STAGES) == stages["GSHT_STAGE_COUNT"]
    for i, name in enumerate(bench.STAGES):
        assert stages[f"GSHT_STAGE_{name.upper()}"] == i, name


def test_bench_stages_are_the_package_stages():
    import gshtrans_b200 as g

    assert tuple(bench.STAGES) == g.STAGES
