"""bench.py's clock sampler against a stand-in nvidia-smi (CPU only).

The sampler starts nvidia-smi before the timed region and drops its first
sample (taken before timing starts); the summary gives the median SM clock
under load, the maximum and the active throttle reasons of the samples
taken while it ran.  The stand-in prints the query's CSV rows at the -lms
interval: the first row is marked by a clock the summary must not see.
"""
import os
import stat
import sys
import textwrap
import time

from conftest import REPO

FAKE = textwrap.dedent("""\
    #!{py}
    import sys, time
    rows = [("111", "Not Active"), ("1965", "Not Active"), ("1950", "Not Active"), ("1965", "Active")]
    for k, (mhz, cap) in enumerate(rows):
        print(f"{{mhz}}, 1965, 900.00, Not Active, Not Active, Not Active, {{cap}}", flush=True)
        time.sleep(0.2)
    time.sleep(30)
""")


def test_clock_sampler_drops_the_pre_timing_sample(tmp_path, monkeypatch):
    exe = tmp_path / "nvidia-smi"
    exe.write_text(FAKE.format(py=sys.executable))
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ.get('PATH', '')}")
    sys.path.insert(0, REPO)
    import bench
    clk = bench.Clocks(0)
    clk.__enter__()            # returns once the first sample has been read
    time.sleep(1.0)            # the "timed region"
    clk.__exit__(None, None, None)
    s = clk.summary()
    assert s["samples"] == 3
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_sampler_without_nvidia_smi(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    sys.path.insert(0, REPO)
    import bench
    clk = bench.Clocks(0)
    clk.__enter__()
    clk.__exit__(None, None, None)
    assert clk.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
