"""bench.py's clock sampler against a stand-in nvidia-smi (CPU; no GPU and no real nvidia-smi needed).

The stand-in takes one sample every 0.05 s (its SM-clock field is the sample number) and, like a
block-buffered nvidia-smi writing to a file, flushes them four at a time, so samples taken before
``mark()`` can reach the file after it.  It also logs each sample's number and epoch time to a side
file, so the test knows which sample was the first one taken inside the timed region.
"""

import importlib.util
import os
import stat
import time

HERE = os.path.dirname(os.path.abspath(__file__))
FAKE = """#!/bin/bash
i=0
buf=""
while true; do
  i=$((i + 1))
  now=$(date +"%s.%3N|%Y/%m/%d %H:%M:%S.%3N")
  echo "$i ${now%%|*}" >> "$FAKE_SMI_LOG"
  buf="$buf${now##*|}, 0, $i, 1965, 500.0, 0x0, Not Active, Not Active, Not Active, Active
"
  if [ $((i % 4)) -eq 0 ]; then printf "%s" "$buf"; buf=""; fi
  sleep 0.05
done
"""


def _bench_module():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(os.path.dirname(HERE), "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _first_sample_at_or_after(log, t):
    for line in open(log):
        i, ts = line.split()
        if float(ts) >= t:
            return int(i)
    return None


def test_clock_sampler_keeps_only_samples_taken_in_the_timed_region(tmp_path, monkeypatch):
    exe = tmp_path / "nvidia-smi"
    exe.write_text(FAKE)
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    log = tmp_path / "samples.log"
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    monkeypatch.setenv("FAKE_SMI_LOG", str(log))
    bench = _bench_module()

    c = bench.ClockSampler(0)
    c.start()  # returns once the first (buffered) samples exist
    time.sleep(0.33)  # samples before the region, some still unflushed at the mark
    c.mark()
    time.sleep(0.4)
    out = c.stop()
    assert out is not None and "note" not in out
    assert out["samples"] >= 2
    first = _first_sample_at_or_after(log, c.mark_time)
    assert first is not None
    # the earliest sample counted is the first one taken at or after the mark; none from before it
    assert out["sm_min_mhz"] == first
    assert out["sm_max_mhz"] == 1965.0 and out["reasons"] == ["sw_power_cap"]


def test_clock_sampler_falls_back_to_the_last_sample_before_a_short_region(tmp_path, monkeypatch):
    exe = tmp_path / "nvidia-smi"
    exe.write_text(FAKE)
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    monkeypatch.setenv("FAKE_SMI_LOG", str(tmp_path / "samples.log"))
    bench = _bench_module()
    c = bench.ClockSampler(0)
    c.start()
    time.sleep(0.3)
    c.mark()
    c.mark_time += 10**6  # as if the region ended before the next sample was taken
    out = c.stop()
    assert out is not None and out["samples"] == 1 and "note" in out
