"""CPU: bench.py's clock sampler reads NVML every 10 ms from a thread during a timed region and maps
the clocks-event reason bits to the names the bench line reports; without NVML it falls back to
nvidia-smi.  A fake pynvml stands in for the library."""
import importlib.util
import os
import sys
import time
import types

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _fake_nvml(reasons, fail_init=False, bus_ok=True):
    nv = types.ModuleType("pynvml")
    nv.NVML_CLOCK_SM = 1
    nv.calls = {"shutdown": 0, "bus": None, "index": None}

    def init():
        if fail_init:
            raise RuntimeError("NVML Shared Library Not Found")
    nv.nvmlInit = init
    nv.nvmlShutdown = lambda: nv.calls.__setitem__("shutdown", nv.calls["shutdown"] + 1)

    def by_bus(b):
        nv.calls["bus"] = b
        if not bus_ok:
            raise RuntimeError("not found")
        return "h"
    nv.nvmlDeviceGetHandleByPciBusId = by_bus
    nv.nvmlDeviceGetHandleByIndex = lambda i: nv.calls.__setitem__("index", i) or "h"
    nv.nvmlDeviceGetMaxClockInfo = lambda h, c: 1965
    clocks = iter([1965, 1965, 1950] + [1965] * 10000)
    nv.nvmlDeviceGetClockInfo = lambda h, c: next(clocks)
    nv.nvmlDeviceGetCurrentClocksEventReasons = lambda h: reasons
    return nv


def _run(monkeypatch, nv, **kw):
    monkeypatch.setitem(sys.modules, "pynvml", nv)
    c = _bench().Clocks(0, **kw)
    c.start()
    time.sleep(0.15)
    return c.stop()


def test_nvml_samples_and_reasons(monkeypatch):
    nv = _fake_nvml(0x4 | 0x1)  # sw_power_cap and gpu_idle (not reported)
    r = _run(monkeypatch, nv, pci_bus_id="00000000:1B:00.0")
    assert r["samples"] >= 5 and r["source"].startswith("nvml")
    assert r["sm_mhz"] == 1965.0 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == ["sw_power_cap"]
    assert nv.calls["bus"] == "00000000:1B:00.0" and nv.calls["shutdown"] == 1


def test_nvml_slowdown_bits(monkeypatch):
    r = _run(monkeypatch, _fake_nvml(0x8 | 0x20 | 0x40))
    assert r["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]


def test_nvml_index_when_bus_unknown(monkeypatch):
    nv = _fake_nvml(0, bus_ok=False)
    r = _run(monkeypatch, nv, pci_bus_id="00000000:99:00.0")
    assert nv.calls["index"] == 0 and r["reasons"] == [] and r["samples"] >= 5


def test_falls_back_without_nvml(monkeypatch):
    monkeypatch.setenv("PATH", "/nonexistent")
    r = _run(monkeypatch, _fake_nvml(0, fail_init=True))
    assert r["sm_mhz"] is None and r["reasons"] == ["nvidia-smi unavailable"]


def _fake_smi(tmp_path, monkeypatch):
    """An nvidia-smi on PATH that prints two CSV rows (one power-capped) and waits to be terminated."""
    exe = tmp_path / "nvidia-smi"
    exe.write_text("#!/bin/sh\n"
                   "echo '0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active'\n"
                   "echo '0, 1800, 1965, 990.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active'\n"
                   "exec sleep 30\n")
    exe.chmod(0o755)
    monkeypatch.setenv("PATH", str(tmp_path) + os.pathsep + os.environ["PATH"])


def test_nvidia_smi_when_nvml_has_no_samples(monkeypatch, tmp_path):
    _fake_smi(tmp_path, monkeypatch)
    nv = _fake_nvml(0)

    def broken(h, c):
        raise RuntimeError("GPU is lost")
    nv.nvmlDeviceGetClockInfo = broken
    r = _run(monkeypatch, nv)
    assert r["source"].startswith("nvidia-smi") and r["samples"] == 2
    assert r["sm_mhz"] == (1965 + 1800) / 2 and r["sm_max_mhz"] == 1965 and r["reasons"] == ["sw_power_cap"]


def test_both_samplers_reported(monkeypatch, tmp_path):
    _fake_smi(tmp_path, monkeypatch)
    r = _run(monkeypatch, _fake_nvml(0))
    assert r["source"].startswith("nvml") and r["nvidia_smi"]["samples"] == 2
