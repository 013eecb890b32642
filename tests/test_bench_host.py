"""Host logic of bench.py that needs no GPU: the clock sampler's parsing of
nvidia-smi's output (median SM clock, maximum, active throttle reasons),
driven by a stand-in nvidia-smi on PATH."""
import os
import stat
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _fake_smi(tmp_path, lines):
    """an nvidia-smi that prints the next of `lines` on every call"""
    data = tmp_path / "lines.txt"
    data.write_text("\n".join(lines) + "\n")
    count = tmp_path / "count.txt"
    count.write_text("0")
    exe = tmp_path / "nvidia-smi"
    exe.write_text(f"""#!{sys.executable}
import sys
lines = open({str(data)!r}).read().splitlines()
k = int(open({str(count)!r}).read())
open({str(count)!r}, "w").write(str(k + 1))
print(lines[min(k, len(lines) - 1)])
""")
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    return str(tmp_path)


def _sample(monkeypatch, path, seconds=1.0):
    monkeypatch.setenv("PATH", path + os.pathsep + os.environ.get("PATH", ""))
    s = bench.ClockSampler(0)
    s.start()
    time.sleep(seconds)
    return s.stop()


def test_clock_sampler_median_max_and_no_reason(tmp_path, monkeypatch):
    lines = ["1965, 1965, 700.5, Not Active, Not Active, Not Active, Not Active",
             "1950, 1965, 710.0, Not Active, Not Active, Not Active, Not Active",
             "1965, 1965, 705.0, Not Active, Not Active, Not Active, Not Active"]
    r = _sample(monkeypatch, _fake_smi(tmp_path, lines))
    assert r["samples"] >= 2
    assert r["sm_max_mhz"] == 1965.0
    assert 1950.0 <= r["sm_mhz"] <= 1965.0
    assert r["reasons"] == []


def test_clock_sampler_reports_active_reasons(tmp_path, monkeypatch):
    lines = ["1300, 1965, 1000.0, Not Active, Not Active, Not Active, Active",
             "1290, 1965, 999.0, Not Active, Active, Not Active, Active"]
    r = _sample(monkeypatch, _fake_smi(tmp_path, lines))
    assert r["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert r["sm_mhz"] < 1400


def test_clock_sampler_without_nvidia_smi_says_unsampled(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))  # nothing named nvidia-smi there
    s = bench.ClockSampler(0)
    s.start()
    time.sleep(0.3)
    r = s.stop()
    assert r["reasons"] == ["unsampled"] and r["sm_mhz"] is None
