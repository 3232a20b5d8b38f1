"""The bench's clock sampler against a fake NVML (no GPU, read-only queries):
samples are taken while the timed region runs, the clock-event reason bits map to
the throttle-reason names that mark a measurement as slowed down, and a failing
query is reported, not swallowed."""
import sys
import time
import types

import pytest


def fake_nvml(bits, fail=False, fail_after=None):
    m = types.ModuleType("pynvml")
    m.NVML_CLOCK_SM = 1
    m.nvmlInit = lambda: None
    m.nvmlDeviceGetHandleByUUID = lambda u: "h"
    m.nvmlDeviceGetHandleByIndex = lambda i: "h"
    m.nvmlDeviceGetMaxClockInfo = lambda h, c: 1965
    m.nvmlDeviceGetClockInfo = lambda h, c: 1800

    calls = [0]

    def reasons(h):
        calls[0] += 1
        if fail or (fail_after is not None and calls[0] > fail_after):
            raise RuntimeError("query failed")
        return bits

    m.nvmlDeviceGetCurrentClocksThrottleReasons = reasons
    return m


@pytest.mark.parametrize("bits,names", [(0, []), (0x4, ["sw_power_cap"]), (0x8 | 0x40, ["hw_slowdown",
                                                                                       "hw_thermal_slowdown"]),
                                        (0x20, ["sw_thermal_slowdown"]), (0x1, [])])
def test_clock_reasons_from_nvml_bits(monkeypatch, bits, names):
    import bench

    monkeypatch.setitem(sys.modules, "pynvml", fake_nvml(bits))
    with bench.Clocks(0) as clk:
        time.sleep(0.05)
    s = clk.summary()
    assert s["source"] == "nvml" and s["samples"] >= 2
    assert s["sm_mhz"] == 1800 and s["sm_max_mhz"] == 1965
    assert s["reasons"] == sorted(names)


def test_clock_query_failure_is_reported(monkeypatch):
    import bench

    monkeypatch.setitem(sys.modules, "pynvml", fake_nvml(0, fail=True))
    with bench.Clocks(0) as clk:
        time.sleep(0.02)
    s = clk.summary()
    assert s["reasons"] == ["unsampled"] and "query failed" in s["error"]


def test_clock_query_failure_after_samples_is_reported(monkeypatch):
    """A query that fails part-way through the region: the samples taken before it are
    kept, and the error is reported beside them (the reasons may be incomplete)."""
    import bench

    monkeypatch.setitem(sys.modules, "pynvml", fake_nvml(0x4, fail_after=3))
    with bench.Clocks(0) as clk:
        time.sleep(0.1)
    s = clk.summary()
    assert s["samples"] == 3 and s["reasons"] == ["sw_power_cap"]
    assert "query failed" in s["error"]
