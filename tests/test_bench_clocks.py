"""The bench's clock record: samples taken inside the timed region by their own timestamps, the
nearest three when the region is shorter than the sampling interval, and throttle reasons.
nvidia-smi is replaced by a script printing lines in its CSV query format."""

from __future__ import annotations

import sys
import time
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402

FAKE = """#!{python}
import datetime, sys, time
while True:
    now = datetime.datetime.now().strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    print(now + ", 1830, 1965, Not Active, Not Active, Not Active, {cap}", flush=True)
    time.sleep(0.05)
"""


def fake_smi(tmp_path: Path, cap: str = "Not Active") -> str:
    p = tmp_path / f"fake-smi-{cap.replace(' ', '-')}"
    p.write_text(FAKE.format(python=sys.executable, cap=cap))
    p.chmod(0o755)
    return str(p)


def test_samples_inside_the_region(tmp_path):
    c = bench.ClockSampler(0, command=fake_smi(tmp_path)).start()
    assert c.lines, "the sampler waits for its first sample"
    time.sleep(0.1)
    t0 = time.time()
    time.sleep(0.4)
    c.mark(t0, time.time())
    time.sleep(0.1)
    c.stop()
    s = c.summary()
    assert s["in_region"] >= 3 and s["samples"] == s["in_region"] and s["slack_ms"] == 0.0
    assert s["sm_mhz"] == 1830.0 and s["sm_max_mhz"] == 1965.0 and s["reasons"] == []
    assert s["window_samples"] > s["samples"]


def test_short_region_takes_the_nearest_three(tmp_path):
    c = bench.ClockSampler(0, command=fake_smi(tmp_path, "Active")).start()
    time.sleep(0.2)
    t0 = time.time()
    c.mark(t0, t0 + 0.001)
    time.sleep(0.2)
    c.stop()
    s = c.summary()
    assert s["samples"] == 3 and s["in_region"] <= 1
    assert 0.0 < s["slack_ms"] < 1000.0  # about 50-100 ms; loose for a loaded host
    assert s["reasons"] == ["sw_power_cap"] and s["window_reasons"] == ["sw_power_cap"]


def test_missing_tool_gives_an_empty_record():
    c = bench.ClockSampler(0, command="/nonexistent/nvidia-smi").start()
    c.mark(0.0, 1.0)
    c.stop()
    assert c.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "in_region": None,
                           "slack_ms": None, "window_samples": 0, "window_reasons": []}


@pytest.mark.parametrize("stamp", ["2026/12/03 19:05:12.345", "2026/12/03 19:05:12"])
def test_timestamp_formats(stamp):
    assert bench.ClockSampler._when(stamp) is not None
    assert bench.ClockSampler._when("not a time") is None
