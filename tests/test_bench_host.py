"""Host-side parts of the benchmark (no GPU): the reference arm's JSON line,
timed from the reference's own step (oracle/_ref) or, without it, from the
C restatement of the same step; the clock sampler's reading of nvidia-smi;
and the rule that re-measures a timing slowed by the hardware."""
import io
import json
import os
import sys
import time
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class Args:
    gpus, steps, warmup = 1, 1, 3


@pytest.mark.skipif(bench.reference_binary() is None,
                    reason="reference oracle not built (make -C oracle)")
def test_reference_arm_prints_one_line_of_the_benchmark_format(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    out = io.StringIO()
    with redirect_stdout(out):
        assert bench.reference_arm(Args()) == 0
    lines = [l for l in out.getvalue().splitlines() if l.strip()]
    assert len(lines) == 1
    r = json.loads(lines[0])
    assert r["impl"] == "reference" and r["metric"] == bench.METRIC and r["unit"] == bench.UNIT
    assert r["value"] > 0 and r["higher_is_better"] is True and r["warmup"] >= 3
    cb = r["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == r["value"]
    assert r["e2e"] == {"value": r["value"], "unit": r["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert "workload" in r["config"]


def test_port_baseline_times_the_c_restatement(monkeypatch):
    monkeypatch.setattr(bench, "reference_binary", lambda: None)
    rate, sec, upd, kind = bench.run_reference(32, 4, 3, 1)
    assert kind == "port" and upd == 32 * 32 and sec > 0 and rate == upd / sec


def test_slowed_timing_is_measured_once_more():
    runs = []

    def timed(reasons):
        def f():
            runs.append(1)
            return 1.0 + len(runs), {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0,
                                     "reasons": reasons if len(runs) == 1 else []}
        return f

    ident = lambda x: x  # noqa: E731  (one rank)
    for reasons, again in ((["hw_slowdown"], True), (["sw_thermal_slowdown"], True),
                           (["sw_power_cap"], False), ([], False)):
        runs.clear()
        ms, clocks, remeasured = bench.timed_with_retry(timed(reasons), ident)
        assert remeasured is again and len(runs) == 1 + again
        assert ms == 1.0 + len(runs)
    # another rank's slowdown makes every rank measure again
    runs.clear()
    _, _, remeasured = bench.timed_with_retry(timed([]), lambda x: max(x, 1.0))
    assert remeasured and len(runs) == 2
    assert not bench.clock_rejected(None)


def test_clock_sampler_reads_clocks_and_reasons(tmp_path, monkeypatch):
    """The sampler's reading of nvidia-smi's CSV, with a stand-in nvidia-smi on
    PATH: median SM clock over the loaded samples, the maximum, and the
    active slowdown reasons by name."""
    fake = tmp_path / "nvidia-smi"
    fake.write_text("#!/bin/sh\n"
                    "echo '0, 1965, 1965, 700.0, 0x4, Not Active, Not Active, Not Active, Active'\n"
                    "echo '0, 1950, 1965, 710.0, 0x4, Not Active, Not Active, Not Active, Active'\n"
                    "echo '0, 345, 1965, 90.0, 0x0, Not Active, Not Active, Not Active, Not Active'\n"
                    "echo '0, 1800, 1965, 900.0, 0x8, Active, Not Active, Not Active, Not Active'\n"
                    "echo 'garbage line'\n"
                    "sleep 5\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}:{os.environ['PATH']}")
    s = bench.ClockSampler(0)
    s.start()
    deadline = time.monotonic() + 10
    while time.monotonic() < deadline:  # the stand-in has written its lines
        with open(s.path) as f:
            if f.read().count("\n") >= 5:
                break
        time.sleep(0.01)
    c = s.stop()
    assert c["samples"] == 4 and c["sm_max_mhz"] == 1965.0
    assert c["sm_mhz"] == 1950.0  # median of the three loaded samples; idle 345 MHz left out
    assert c["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert bench.clock_rejected(c)
