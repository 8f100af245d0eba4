"""The benchmark's clock record, read through a fake NVML on the CPU: the
median SM clock, the union of clock-event reasons over the samples, and the
device looked up by PCI bus id with the CUDA index as fallback.  Nothing
here touches a GPU or sets a clock."""
import importlib.util
import os
import sys
import time
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _fake_nvml(clocks, masks, by_bus=True):
    nv = types.ModuleType("pynvml")
    nv.NVML_CLOCK_SM = 1
    nv.nvmlClocksEventReasonSwPowerCap = 0x4
    nv.nvmlClocksEventReasonHwSlowdown = 0x8
    nv.nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nv.nvmlClocksEventReasonHwThermalSlowdown = 0x40
    state = {"i": 0, "lookups": []}

    def nxt(seq):
        return seq[min(state["i"], len(seq) - 1)]

    def init():
        state["init"] = True

    def by_pci(bus):
        state["lookups"].append(("bus", bus))
        if not by_bus:
            raise RuntimeError("not found")
        return "h"

    def by_index(i):
        state["lookups"].append(("index", i))
        return "h"

    def clock(h, kind):
        v = nxt(clocks)
        state["i"] += 1
        return v

    nv.nvmlInit = init
    nv.nvmlShutdown = lambda: None
    nv.nvmlDeviceGetHandleByPciBusId = by_pci
    nv.nvmlDeviceGetHandleByIndex = by_index
    nv.nvmlDeviceGetClockInfo = clock
    nv.nvmlDeviceGetMaxClockInfo = lambda h, k: 1965
    nv.nvmlDeviceGetPowerUsage = lambda h: 950000
    nv.nvmlDeviceGetCurrentClocksEventReasons = lambda h: nxt(masks)
    return nv, state


@pytest.mark.parametrize("by_bus", [True, False])
def test_nvml_samples_median_and_reasons(monkeypatch, by_bus):
    bench = _bench()
    nv, state = _fake_nvml([1965, 1900, 1965, 1965], [0x0, 0x4, 0x0, 0x0], by_bus=by_bus)
    monkeypatch.setitem(sys.modules, "pynvml", nv)
    c = bench.Clocks(0)
    monkeypatch.setattr(c, "_bus_id", lambda: "00000000:18:00.0")
    c.start()
    time.sleep(0.1)
    rec = c.stop()
    assert rec["source"] == "nvml"
    assert rec["samples"] >= 3
    assert rec["sm_max_mhz"] == 1965
    assert rec["sm_min_mhz"] == 1900
    assert rec["sm_mhz"] == 1965
    assert rec["reasons"] == ["sw_power_cap"]
    assert rec["power_w_median"] == 950.0
    assert state["lookups"][0] == ("bus", "00000000:18:00.0")
    if not by_bus:
        assert state["lookups"][1] == ("index", 0)


def test_slowdown_reasons_are_reported(monkeypatch):
    bench = _bench()
    nv, _ = _fake_nvml([1500], [0x8 | 0x40 | 0x20])
    monkeypatch.setitem(sys.modules, "pynvml", nv)
    c = bench.Clocks(0)
    c.start()
    rec = c.stop()
    assert rec["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]
    assert rec["sm_mhz"] == 1500


def test_no_nvml_no_smi_gives_no_record(monkeypatch):
    bench = _bench()
    broken = types.ModuleType("pynvml")

    def fail():
        raise RuntimeError("no driver")

    broken.nvmlInit = fail
    monkeypatch.setitem(sys.modules, "pynvml", broken)

    def no_smi(*a, **k):
        raise OSError("nvidia-smi not found")

    monkeypatch.setattr(bench.subprocess, "Popen", no_smi)
    c = bench.Clocks(0)
    c.start()
    assert c.stop() is None
