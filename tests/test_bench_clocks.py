"""CPU: the bench's clock sampler (read-only NVML queries during the timed
region) against a fake NVML module: it picks the reasons call that works,
decodes the throttle bits, falls back to nvidia-smi when NVML is missing, and
says why when nothing could be sampled. No GPU and no real NVML involved."""
import os
import sys
import time
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def fake_nvml(event_reasons=None, throttle_reasons=0, sm=1950, max_sm=1965):
    nv = types.ModuleType("pynvml")
    nv.NVML_CLOCK_SM = 1
    nv.nvmlClocksEventReasonHwSlowdown = 0x8
    nv.nvmlClocksEventReasonHwThermalSlowdown = 0x40
    nv.nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nv.nvmlClocksEventReasonSwPowerCap = 0x4
    nv.nvmlInit = lambda: None
    nv.nvmlShutdown = lambda: None
    nv.nvmlDeviceGetHandleByIndex = lambda i: ("gpu", i)
    nv.nvmlDeviceGetMaxClockInfo = lambda h, c: max_sm
    nv.nvmlDeviceGetClockInfo = lambda h, c: sm

    def event(h):
        if event_reasons is None:
            raise RuntimeError("Function Not Found")
        return event_reasons

    nv.nvmlDeviceGetCurrentClocksEventReasons = event
    nv.nvmlDeviceGetCurrentClocksThrottleReasons = lambda h: throttle_reasons
    return nv


def sample_for(monkeypatch, nv, seconds=0.06):
    if nv is None:
        monkeypatch.setitem(sys.modules, "pynvml", None)  # import fails
    else:
        monkeypatch.setitem(sys.modules, "pynvml", nv)
    c = bench.ClockSampler(0)
    c.start()
    time.sleep(seconds)
    return c.stop()


def test_event_reasons_are_decoded(monkeypatch):
    out = sample_for(monkeypatch, fake_nvml(event_reasons=0x4 | 0x40))
    assert out["source"] == "nvml" and out["samples"] >= 1
    assert out["sm_mhz"] == 1950 and out["sm_max_mhz"] == 1965
    assert out["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]


def test_throttle_reasons_call_is_the_fallback(monkeypatch):
    out = sample_for(monkeypatch, fake_nvml(event_reasons=None, throttle_reasons=0))
    assert out["source"] == "nvml" and out["samples"] >= 1
    assert out["reasons"] == []


def test_without_nvml_the_failure_is_reported(monkeypatch):
    monkeypatch.setattr(bench.subprocess, "run", lambda *a, **k: (_ for _ in ()).throw(FileNotFoundError("nvidia-smi")))
    out = sample_for(monkeypatch, None)
    assert out["source"] == "nvidia-smi"
    assert out["reasons"] == ["unsampled"] and out["sm_mhz"] is None
    assert "nvml" in out["note"] or "nvidia-smi" in out["note"]
