"""bench.py's clock sampler against a stand-in nvidia-smi (CPU; no GPU and no real nvidia-smi needed).

The stand-in prints one CSV sample every 0.05 s with the sample number as the SM clock, so the test
can tell which samples the sampler attributed to the timed region: only those written after
``mark()``, even when the region is short, and the last earlier sample when none fell inside it.
"""

import importlib.util
import os
import stat
import time

HERE = os.path.dirname(os.path.abspath(__file__))
FAKE = """#!/bin/sh
i=0
while true; do
  i=$((i + 1))
  echo "0, $i, 1965, 500.0, 0x0, Not Active, Not Active, Not Active, Active"
  sleep 0.05
done
"""


def _bench_module():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(os.path.dirname(HERE), "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_clock_sampler_keeps_only_the_timed_region(tmp_path, monkeypatch):
    exe = tmp_path / "nvidia-smi"
    exe.write_text(FAKE)
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    bench = _bench_module()

    c = bench.ClockSampler(0)
    c.start()  # returns once the first sample exists
    time.sleep(0.3)  # samples before the region
    c.mark()
    first_in_region = c.mark_line + 1  # the stand-in's clock field is its 1-based sample number
    time.sleep(0.3)
    out = c.stop()
    assert out is not None and "note" not in out
    assert out["samples"] >= 2
    assert out["sm_mhz"] >= first_in_region  # no sample from before the mark
    assert out["sm_max_mhz"] == 1965.0 and out["reasons"] == ["sw_power_cap"]

    c = bench.ClockSampler(0)
    c.start()
    time.sleep(0.2)
    c.mark()
    c.mark_line += 10**6  # as if the region ended before the next sample was written
    out = c.stop()
    assert out is not None and out["samples"] == 1 and "note" in out
