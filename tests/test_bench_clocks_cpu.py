"""bench.py's clock record: nvidia-smi samples parsed, only those inside the
timed region kept, throttle reasons collected (a fake sampler output, no GPU)."""
import datetime
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class _DoneProc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def _line(t, sm, reasons=("Not Active",) * 4):
    stamp = datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    return f"{stamp}, 0, {sm}, 1965, 900.5, 0x0000000000000000, " + ", ".join(reasons) + "\n"


def _sampler(tmp_path, lines, begin, end):
    c = bench.ClockSampler(0)
    c.path = str(tmp_path / "clk.csv")
    with open(c.path, "w") as f:
        f.writelines(lines)
    c.proc = _DoneProc()
    c.t_begin, c.t_end = begin, end
    return c


def test_samples_outside_the_timed_region_are_dropped(tmp_path):
    t = 1.8e9
    lines = [_line(t - 1.0, 1200), _line(t + 0.10, 1965), _line(t + 0.15, 1950), _line(t + 0.20, 1965),
             _line(t + 2.0, 800, ("Not Active", "Active", "Not Active", "Not Active"))]
    out = _sampler(tmp_path, lines, t, t + 0.3).stop()
    assert out["samples"] == 3
    assert out["sm_mhz"] == 1965 and out["sm_max_mhz"] == 1965
    assert out["reasons"] == [] and out["window"] == "timed region"


def test_throttle_reasons_inside_the_region_are_reported(tmp_path):
    t = 1.8e9
    lines = [_line(t + 0.1, 1800, ("Not Active", "Not Active", "Not Active", "Active")),
             _line(t + 0.2, 1700, ("Active", "Not Active", "Not Active", "Not Active"))]
    out = _sampler(tmp_path, lines, t, t + 0.3).stop()
    assert out["samples"] == 2 and out["sm_mhz"] == 1750
    assert out["reasons"] == ["hw_slowdown", "sw_power_cap"]


def test_region_without_samples_falls_back_to_all(tmp_path):
    t = 1.8e9
    out = _sampler(tmp_path, [_line(t - 1.0, 1965), _line(t + 5.0, 1965)], t, t + 0.1).stop()
    assert out["samples"] == 2 and out["window"].startswith("whole sampling")


def test_no_sampler_process():
    assert bench.ClockSampler(0).stop() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
