"""The bench's clock sampler (bench.Clocks) against a stand-in nvidia-smi: a
script on PATH that prints one CSV sample every 50 ms, as `nvidia-smi
--query-gpu=... --format=csv,noheader,nounits -lms N` does.  No GPU."""
from __future__ import annotations

import os
import stat
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402

FAKE = """#!/bin/sh
sleep {startup}
i=0
while [ $i -lt 400 ]; do
  echo "{mhz}, 1965, 612.3, 0x0000000000000004, Not Active, Not Active, Not Active, {cap}"
  i=$((i + 1))
  sleep 0.05
done
"""


def run_with_fake(tmp_path, monkeypatch, mhz, cap, seconds, startup=0.0):
    exe = tmp_path / "nvidia-smi"
    exe.write_text(FAKE.format(mhz=mhz, cap=cap, startup=startup))
    exe.chmod(exe.stat().st_mode | stat.S_IXUSR)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ.get('PATH', '')}")
    with bench.Clocks(0) as c:
        time.sleep(seconds)
    return c.summary


def test_short_region_is_sampled(tmp_path, monkeypatch):
    """A region shorter than a few sampling periods still gets samples: the
    sampler waits for nvidia-smi's first line before the region starts (the
    stand-in takes 0.2 s to start, as the tool takes a moment)."""
    s = run_with_fake(tmp_path, monkeypatch, 1965, "Not Active", 0.12, startup=0.2)
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["samples"] >= 1 and s["reasons"] == []


def test_power_cap_reason_is_reported(tmp_path, monkeypatch):
    s = run_with_fake(tmp_path, monkeypatch, 1320, "Active", 0.3)
    assert s["sm_mhz"] == 1320.0
    assert s["reasons"] == ["sw_power_cap"]


def test_missing_tool_leaves_the_region_unsampled(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    with bench.Clocks(0) as c:
        pass
    assert c.summary == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
