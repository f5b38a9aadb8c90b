"""The bench's clock sampler against a stand-in for nvidia-smi (CPU only): rows
after mark() are the timed-region samples, throttle reasons are parsed, and an
absent tool yields an empty record instead of an error."""
import os
import stat
import sys
import textwrap
import time

import bench

FAKE = textwrap.dedent("""\
    import sys, time
    ms = int(sys.argv[sys.argv.index("-lms") + 1])
    n = 0
    while True:
        n += 1
        cap = "Active" if n % 2 else "Not Active"
        sys.stdout.write("0, %d, 1965, 700.0, 0x4, Not Active, Not Active, Not Active, %s\\n" % (1900 + n % 3, cap))
        sys.stdout.flush()
        time.sleep(ms / 1000.0)
""")


def _fake_tool(tmp_path):
    py = tmp_path / "fake_smi.py"
    py.write_text(FAKE)
    exe = tmp_path / "fake-smi"
    exe.write_text("#!/bin/sh\nexec %s %s \"$@\"\n" % (sys.executable, py))
    exe.chmod(exe.stat().st_mode | stat.S_IXUSR)
    return str(exe)


def _wait_rows(clk, n, limit=10.0):
    t = time.time()
    while len(clk._rows()) < n and time.time() - t < limit:
        time.sleep(0.01)


def test_samples_after_mark_are_reported(tmp_path):
    clk = bench.Clocks(0, interval_ms=10, exe=_fake_tool(tmp_path))
    _wait_rows(clk, 5)                         # the warm-up: sampler running
    clk.mark()
    before = clk.start_row
    _wait_rows(clk, before + 5)                # the timed region
    out = clk.stop()
    assert before >= 5
    assert out["window"] == "timed" and out["samples"] >= 5
    assert out["sm_max_mhz"] == 1965.0 and 1900.0 <= out["sm_mhz"] <= 1902.0
    assert out["reasons"] == ["sw_power_cap"]


def test_short_timed_region_falls_back_to_warm_up_samples(tmp_path):
    clk = bench.Clocks(0, interval_ms=2000, exe=_fake_tool(tmp_path))
    _wait_rows(clk, 1)
    clk.mark()                                 # no sample lands before stop()
    out = clk.stop()
    assert out["samples"] >= 1 and out["window"].startswith("warm-up")
    assert out["sm_mhz"] is not None


def test_missing_tool_gives_empty_record(tmp_path):
    clk = bench.Clocks(0, exe=str(tmp_path / "no-such-tool"))
    clk.mark()
    out = clk.stop()
    assert out == {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
    assert not os.path.exists(tmp_path / "no-such-tool")


def test_no_row_visible_at_mark_is_labelled(tmp_path):
    """output that only appears at exit (a buffered tool): all samples, said so"""
    clk = bench.Clocks(0, interval_ms=10, exe=_fake_tool(tmp_path))
    clk.mark()                                 # before the first row
    clk.start_row = 0
    _wait_rows(clk, 3)
    out = clk.stop()
    assert out["samples"] >= 3 and out["window"].startswith("warm-up and timed")
