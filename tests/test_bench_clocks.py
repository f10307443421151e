"""bench.py's clock record: only samples stamped inside the timed region
count, and the active-reasons bitmask is decoded into reason names (no GPU:
the nvidia-smi lines are synthetic)."""
import datetime
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402


class _Proc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        pass


class _Thread:
    def join(self, timeout=None):
        pass


def _stamp(t):
    return datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]


def _clocks(lines):
    c = bench.Clocks(0)
    c.lines, c.proc, c.t = lines, _Proc(), _Thread()
    return c


def test_region_filter_and_reasons():
    t0 = time.time()
    lines = [
        f"{_stamp(t0 - 2)}, 0, 900, 1965, 90.0, 0x0000000000000001, Not Active, Not Active, Not Active, Not Active",
        f"{_stamp(t0 + 0.1)}, 0, 1800, 1965, 700.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        f"{_stamp(t0 + 0.2)}, 0, 1700, 1965, 760.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        f"{_stamp(t0 + 0.3)}, 0, 1750, 1965, 740.0, 0x0000000000000080, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
        f"{_stamp(t0 + 5)}, 0, 300, 1965, 60.0, 0x0000000000000001, Not Active, Not Active, Not Active, Not Active",
    ]
    r = _clocks(lines).stop(t0, t0 + 1)
    assert r["samples"] == 3
    assert r["sm_mhz"] == 1750.0 and r["sm_max_mhz"] == 1965.0 and r["power_w_max"] == 760.0
    assert r["reasons"] == ["hw_power_brake_slowdown", "sw_power_cap"]  # gpu_idle samples lie outside


def test_no_sampler():
    c = bench.Clocks(0)
    assert c.stop()["reasons"] == ["nvidia-smi unavailable"]
