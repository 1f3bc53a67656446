"""The bench's clock sampler, against a fake nvidia-smi on the PATH (CPU only):
it reports only the samples written inside the load window, and parses the
throttle reasons."""
import importlib.util
import os
import stat
import time

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

FAKE = """#!/bin/sh
# prints one CSV sample every 50 ms: index, sm, max sm, power, active mask,
# hw_slowdown, hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap
n=0
while [ $n -lt 400 ]; do
  echo "0, 1800, 1965, 700.5, 0x0000000000000004, Not Active, Not Active, Not Active, Active"
  n=$((n+1))
  sleep 0.05
done
"""


def load_bench():
    spec = importlib.util.spec_from_file_location("cola_bench", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_clock_window(tmp_path, monkeypatch):
    fake = tmp_path / "nvidia-smi"
    fake.write_text(FAKE)
    fake.chmod(fake.stat().st_mode | stat.S_IXUSR)
    monkeypatch.setenv("PATH", str(tmp_path) + os.pathsep + os.environ.get("PATH", ""))
    bench = load_bench()
    c = bench.Clocks(0)
    c.start()
    assert c.proc is not None and c.lo >= 1  # returned after the first sample
    time.sleep(0.4)
    c.hold()  # no step: just ends the window
    time.sleep(0.3)  # samples after the window are not reported
    r = c.stop()
    assert r is not None
    assert r["sm_mhz"] == 1800.0 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == ["sw_power_cap"]
    assert 3 <= r["samples"] <= 12, r
    assert 0.35 <= r["window_s"] <= 1.5, r


def test_clock_sampler_absent(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))  # no nvidia-smi at all
    bench = load_bench()
    c = bench.Clocks(0)
    c.start()
    c.hold(lambda: None)
    assert c.stop() is None
