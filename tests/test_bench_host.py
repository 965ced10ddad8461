"""Host-side parts of the benchmark (no GPU): the reference arm's JSON line,
timed from the reference's own step (oracle/_ref, its shared-memory MPI mode)
or, without it, from the C restatement of the same step; the clock sampler's reading of nvidia-smi;
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
    gpus, steps, warmup, n = 1, 1, 3, 64


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
    rate, sec, upd, kind, n = bench.run_reference(32, 4, 3, 1)
    assert kind == "port" and n == 32 and upd == 32 * 32 and sec > 0 and rate == upd / sec


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


class FakeNvml:
    """Stand-in for pynvml: one GPU at a given PCI bus id, a scripted clock
    and reason sequence."""
    NVML_CLOCK_SM = 1
    nvmlClocksEventReasonHwSlowdown = 0x8
    nvmlClocksEventReasonHwThermalSlowdown = 0x40
    nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nvmlClocksEventReasonSwPowerCap = 0x4

    def __init__(self, bus_id, script):
        self.bus_id, self.script, self.i, self.asked = bus_id, script, 0, []

    def nvmlInit(self):
        pass

    def nvmlDeviceGetHandleByPciBusId(self, bus):
        self.asked.append(bus)
        if bus != self.bus_id:
            raise RuntimeError("no such GPU")
        return "h"

    def nvmlDeviceGetMaxClockInfo(self, h, clk):
        return 1965

    def nvmlDeviceGetClockInfo(self, h, clk):
        return self.script[min(self.i, len(self.script) - 1)][0]

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        mask = self.script[min(self.i, len(self.script) - 1)][1]
        self.i += 1
        return mask


def test_clock_sampler_reads_nvml_for_the_benchmarks_gpu(monkeypatch):
    """With CUDA_VISIBLE_DEVICES selecting another GPU than NVML's first, the
    sampler asks NVML for the GPU by its PCI bus id; it reports the median
    SM clock of the loaded samples taken inside the timed window, the
    maximum clock and the active slowdown reasons by name."""
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "5")
    fake = FakeNvml("00000000:9A:00.0", [(1965, 0x4), (1950, 0x4), (345, 0x0), (1800, 0x8)])
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    s = bench.ClockSampler(0, bus_id="00000000:9A:00.0", interval_s=0.0005)
    s.start()
    deadline = time.monotonic() + 5
    while fake.i < 4 and time.monotonic() < deadline:
        time.sleep(0.005)
    c = s.stop()
    assert fake.asked == ["00000000:9A:00.0"]
    assert c["source"] == "nvml" and c["sm_max_mhz"] == 1965.0 and c["samples"] >= 4
    assert c["sm_mhz"] >= 1800.0  # loaded samples only; the idle 345 MHz left out
    assert c["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert bench.clock_rejected(c)
    # samples taken outside the timed window do not count
    s.rows = [(s.t0 - 1.0, 900.0, {"hw_slowdown"})] + [(s.t0 + 1e-6, 1965.0, set())]
    c = s.summary()
    assert c["samples"] == 1 and c["reasons"] == [] and c["sm_mhz"] == 1965.0


def test_clock_sampler_falls_back_to_nvidia_smi_by_bus_id(tmp_path, monkeypatch):
    """Without NVML: a stand-in nvidia-smi on PATH records its arguments; the
    sampler selects the GPU by bus id and keeps only the samples stamped
    inside the timed window."""
    import datetime
    monkeypatch.setitem(sys.modules, "pynvml", None)  # import fails
    now = datetime.datetime.now()
    stamp = lambda dt: (now + datetime.timedelta(seconds=dt)).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]  # noqa: E731
    args_file = tmp_path / "args"
    fake = tmp_path / "nvidia-smi"
    fake.write_text("#!/bin/sh\n"
                    f"echo \"$@\" > {args_file}\n"
                    f"echo '{stamp(-60)}, 900, 1965, Active, Not Active, Not Active, Not Active'\n"
                    f"echo '{stamp(0.2)}, 1965, 1965, Not Active, Not Active, Not Active, Active'\n"
                    f"echo '{stamp(0.3)}, 1950, 1965, Not Active, Not Active, Not Active, Active'\n"
                    "echo 'garbage line'\n"
                    "sleep 5\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}:{os.environ['PATH']}")
    s = bench.ClockSampler(0, bus_id="00000000:1B:00.0")
    s.start()
    deadline = time.monotonic() + 10
    while time.monotonic() < deadline:  # the stand-in has written its lines
        with open(s.path) as f:
            if f.read().count("\n") >= 4:
                break
        time.sleep(0.01)
    time.sleep(0.5)  # the region covers the stamps 0.2 s and 0.3 s after start
    c = s.stop()
    assert "--id=00000000:1B:00.0" in args_file.read_text()
    assert c["source"] == "nvidia-smi" and c["samples"] == 2
    assert c["sm_mhz"] == 1957.5 and c["reasons"] == ["sw_power_cap"]
    assert not bench.clock_rejected(c)


def test_spawned_ranks_run_one_job():
    """bench.py --gpus N without a launcher starts N ranks itself: each gets
    RANK, LOCAL_RANK, WORLD_SIZE and a 127.0.0.1 rendezvous, and they form
    one gloo job."""
    code = ("import os, torch, torch.distributed as dist\n"
            "dist.init_process_group('gloo')\n"
            "t = torch.tensor([float(os.environ['RANK']) + 1.0])\n"
            "dist.all_reduce(t)\n"
            "assert t.item() == 3.0 and os.environ['LOCAL_RANK'] == os.environ['RANK']\n"
            "assert os.environ['MASTER_ADDR'] == '127.0.0.1' and dist.get_world_size() == 2\n"
            "dist.destroy_process_group()\n")
    assert bench.spawn_ranks(2, [sys.executable, "-c", code], timeout=120) == [0, 0]
    # a failing rank fails the job
    assert bench.spawn_ranks(2, [sys.executable, "-c", "import os, sys; "
                                 "sys.exit(int(os.environ['RANK']) * 3)"], timeout=60)[1] == 3


def test_launcher_world_size_must_match_gpus(monkeypatch, capsys):
    monkeypatch.setenv("WORLD_SIZE", "4")
    assert bench.main(["--gpus", "2", "--impl", "reference"]) == 2
    assert "WORLD_SIZE=4" in capsys.readouterr().err
