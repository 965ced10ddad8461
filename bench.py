#!/usr/bin/env python
"""Benchmark of the B200 explicit time step (leaf-cell updates per second).

Workload: the flux/stage bandwidth case — a 2048 x 2048 single-level periodic
grid on [0,10]^2 with an isentropic vortex (strength 5) advected at Mach 0.5
and 45 degrees, inviscid, 4-stage low-storage scheme, VanLeer MUSCL, all-speed
Roe flux, CFL 0.5 (dt from the CFL condition every step).  One bench "step" is
one full time step of every leaf cell (4 stages).  Synthetic inputs built on
the host; the state (~470 MB with its stage buffers) is larger than L2, so no
flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas of the case, one per GPU (the single case
does not shard; whole-job throughput = cells x steps x N / max-over-ranks time).
"""
from __future__ import annotations

import argparse
import contextlib
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "Cell-updates/s (B200): FP64 plain vs mixed/batched/learned at |dCl|,|dCd|<1e-3"
UNIT = "cell-updates/s"
N_DEFAULT = 2048
STAGES = 4
# algorithmic bytes per leaf cell per stage, inviscid: read U^(k-1) (32 B),
# read U^n (32 B), write U^(k) (32 B)
BYTES_PER_CELL_STAGE = 96
# host memory of the reference's own run of the 2048^2 case (measured: 18.0 GB
# of shared windows, ~0.25 GB private per rank); smaller grids scale with n^2
REF_SHARED_BYTES_2048 = 18.0e9
REF_RANK_BYTES = 0.3e9
PORT_SAMPLE_N = 512  # the C restatement's sample (one core) when the reference build is absent
BATCH_CASES = 64     # batched workload: independent cases, 50k..800k leaf cells each
REGRID_EVERY = 20    # steps between regrids of the airfoil workloads (learned tagging cost)
NACA_RECORD = os.path.join(ROOT, "tests", "golden", "naca_minmod_s4_n64_l3.npz")
# the plain-method airfoil workload at its stated size (128^2 base + 3 AMR
# levels, 400-point NACA0012, Mach 0.5, 2 deg, Re 5000, minmod, 4 stages,
# CFL 0.5): the reference's mesh, initial state and 1000-step force history
CONFIG1_RECORD = os.path.join(ROOT, "tests", "golden", "naca_minmod_s4_n128_l4.npz")
CONFIG1_HISTORY = os.path.join(ROOT, "tests", "golden", "naca_forces_s1000_n128_l4.npz")
CONFIG1_ENV = {"IB_NX": "128", "IB_LEVELS": "4", "IB_STAGES": "4", "IB_USER_INIT": "0",
               "IB_NPTS": "200"}
F_REF = 0.5 * 1.0 * 0.1  # 0.5 rho_inf u_inf^2 * chord * slab depth (Cl, Cd scale)
# the moving-body workload at its stated size: a NACA0015 pitching about its
# quarter chord (5 deg, k = 0.1, mean 0), Mach 0.2, Re 1e4, 256^2 base grid on
# [0,30]^2 + 5 AMR levels tracking the body and wake (~1.58 M leaf cells),
# regrid every 20 steps; built and moved by the reference's own host code
# the batched airfoil workload: 64 independent NACA0012 / NACA0015 cases
# (alternating) from a seeded generator; the first CONFIG4_DEFAULT_CASES run by
# default (the host meshes come from the reference's own mesh generation)
CONFIG4_CASES = 64
CONFIG4_DEFAULT_CASES = 16
# leaf cells per base cell of the airfoil mesh by mesh level count (the base
# grid and its AMR levels; measured on the reference's 256^2-base meshes of
# this case family): base side = sqrt(target / f)
CONFIG4_LEAF_FACTOR = {3: 1.81, 4: 2.71, 5: 3.95, 6: 6.22}
CONFIG3_ENV = {"IB_NX": "256", "IB_LEVELS": "6", "IB_STAGES": "4", "IB_USER_INIT": "0",
               "IB_NPTS": "400", "IB_REGRID_EVERY": "20", "IB_PITCH_K": "0.1",
               "IB_FORCES": "1"}


def load_pkg():
    name = "immsered_boundary_b200"
    if name in sys.modules:
        return sys.modules[name]
    pdir = os.path.join(ROOT, "immsered-boundary_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pdir, "__init__.py"),
                                                  submodule_search_locations=[pdir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


@contextlib.contextmanager
def near_gpu_cores(device: int = 0):
    """Run the block on the host cores next to the GPU (NVML's CPU affinity
    of the device, i.e. its NUMA node), so that pinned buffers allocated and
    first touched inside it live in that node's memory and the copies do
    not cross the socket link; the previous affinity returns afterwards.
    Yields the cores used, or None when the affinity is unknown (no
    change)."""
    old = os.sched_getaffinity(0)
    cpus = None
    try:
        import pynvml
        import torch
        pr = torch.cuda.get_device_properties(device)
        pynvml.nvmlInit()
        h = pynvml.nvmlDeviceGetHandleByPciBusId(
            f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0")
        words = pynvml.nvmlDeviceGetCpuAffinity(h, (os.cpu_count() + 63) // 64)
        cpus = {64 * i + b for i, w in enumerate(words) for b in range(64) if (w >> b) & 1} & old
    except Exception:
        cpus = None
    if cpus and cpus != old:
        os.sched_setaffinity(0, cpus)
    try:
        yield sorted(cpus) if cpus else None
    finally:
        if cpus and cpus != old:
            os.sched_setaffinity(0, old)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(key="stage_kernel_fp64_vortex2048"):
    """DRAM bytes per stage launch (dram__bytes_read.sum + dram__bytes_write.sum
    of one ncu capture) from profiles/roofline_traffic.json, if recorded."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    try:
        with open(p) as f:
            return float(json.load(f)[key]["dram_bytes_per_launch"])
    except (OSError, KeyError, ValueError, TypeError):
        return None


def pci_bus_id(device: int):
    """PCI bus id of a CUDA device (CUDA ordinals follow CUDA_VISIBLE_DEVICES
    and CUDA_DEVICE_ORDER; NVML and nvidia-smi index GPUs their own way, so
    the bus id is the key both understand), or None when unknown."""
    try:
        import torch
        pr = torch.cuda.get_device_properties(device)
        return f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
    except Exception:
        return None


REASON_NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")


class ClockSampler:
    """SM clock and clock-event reasons of the benchmark's GPU, sampled
    during the timed region only.

    NVML is polled from a thread about every millisecond between start() and
    stop(), so that a timed region of a few milliseconds still gets samples;
    the GPU is found by its PCI bus id.  Without NVML, nvidia-smi is polled
    every 20 ms (the same bus id as --id) and only its samples stamped
    inside the region count."""

    def __init__(self, device: int, bus_id: str | None = None, interval_s: float = 0.001):
        self.bus_id = bus_id if bus_id is not None else pci_bus_id(device)
        self.interval = interval_s
        self.rows = []  # (host time, sm MHz, set of reason names)
        self.max_mhz = None
        self._thread = None
        self._stop = None
        self._proc = None
        self.path = None
        self.error = None
        self.t0 = self.t1 = None

    # ---- NVML
    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        if self.bus_id is None:
            raise RuntimeError("no PCI bus id")
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(self.bus_id)

    def _poll(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        while not self._stop.is_set():
            t = time.perf_counter()
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
            except Exception as e:  # noqa: BLE001
                self.error = f"nvmlDeviceGetClockInfo: {e}"
                break
            try:
                mask = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                reasons = {n for n, b in bits.items() if mask & b}
            except Exception as e:  # noqa: BLE001
                self.error = f"nvmlDeviceGetCurrentClocksEventReasons: {e}"
                reasons = {"unknown"}
            self.rows.append((t, mhz, reasons))
            self._stop.wait(self.interval)

    def start(self):
        import threading
        self.rows = []
        self.error = None
        self._stop = threading.Event()
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self._thread.start()
            # the window opens once the poller has its first sample
            t = time.perf_counter()
            while not self.rows and self._thread.is_alive() and time.perf_counter() - t < 0.5:
                time.sleep(0.0002)
        except Exception as e:  # noqa: BLE001
            self.error = f"nvml: {e}"
            self._thread = None
            self._start_smi()
            time.sleep(0.1)  # nvidia-smi's first sample
        self.t0 = time.perf_counter()

    # ---- nvidia-smi fallback
    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def _start_smi(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        ident = [f"--id={self.bus_id}"] if self.bus_id else []
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", *ident, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self._proc = None

    def _read_smi(self):
        import datetime
        # nvidia-smi stamps in local wall-clock time: map onto perf_counter
        off = time.time() - time.perf_counter()
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                mhz, mx = float(parts[1]), float(parts[2])
            except ValueError:
                continue
            self.max_mhz = max(self.max_mhz or 0.0, mx)
            self.rows.append((ts - off, mhz, {n for n, f in zip(REASON_NAMES, parts[3:7])
                                              if f.lower() == "active"}))

    def stop(self):
        self.t1 = time.perf_counter()
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)
        elif self._proc is not None:
            time.sleep(0.05)  # a last sample stamped after the region
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
            self._read_smi()
            os.unlink(self.path)
        else:
            return None
        return self.summary()

    def summary(self):
        inside = [r for r in self.rows if self.t0 <= r[0] <= self.t1]
        where = "inside the timed region"
        if not inside:
            # a region shorter than the poll period: the samples that bracket it
            before = [r for r in self.rows if r[0] < self.t0][-1:]
            after = [r for r in self.rows if r[0] > self.t1][:1]
            inside = before + after
            where = "nearest samples before and after the timed region"
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0,
                    "window_ms": (self.t1 - self.t0) * 1e3, "error": self.error or "no samples",
                    "gpu": self.bus_id}
        mx = self.max_mhz or max(r[1] for r in inside)
        loaded = [r[1] for r in inside if r[1] > 0.5 * mx] or [r[1] for r in inside]
        reasons = sorted(set().union(*(r[2] for r in inside)))
        out = {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": reasons,
               "samples": len(inside), "window_ms": (self.t1 - self.t0) * 1e3,
               "source": "nvml" if self._thread is not None else "nvidia-smi",
               "sampled": where, "gpu": self.bus_id}
        if self.error:
            out["error"] = self.error
        return out


# clock-event reasons that make a timing invalid (sw_power_cap is kept and noted)
BAD_CLOCK_REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown")


def clock_rejected(clocks) -> bool:
    return bool(clocks) and any(r in BAD_CLOCK_REASONS for r in clocks.get("reasons", ()))


def timed_with_retry(timed, reduce_max):
    """timed() -> (ms, clocks).  When the clock record (rank 0's) shows a
    hardware or thermal slowdown, measure once more; the decision goes
    through reduce_max so that every rank takes the same steps.  Returns
    (ms, clocks, remeasured)."""
    ms, clocks = timed()
    if reduce_max(1.0 if clock_rejected(clocks) else 0.0) > 0.0:
        ms, clocks = timed()
        return ms, clocks, True
    return ms, clocks, False


def reference_binary():
    p = os.path.join(ROOT, "oracle", "_ref", "ref_vortex_vanleer")
    return p if os.path.exists(p) and os.access(p, os.X_OK) else None


def host_cores() -> int:
    """Host cores this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def avail_bytes() -> float:
    try:
        return float(os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE"))
    except (ValueError, OSError):
        return float("inf")


def host_workers(per_worker_bytes: float) -> int:
    """Concurrent host processes of `per_worker_bytes` each that fit the
    host cores and the available memory."""
    return max(1, min(host_cores(), int(0.7 * avail_bytes() // per_worker_bytes)))


def run_reference_mpi(binary: str, env_case: dict, steps: int, warmup: int, ranks: int,
                      timeout: float = 1800.0):
    """One run of a reference oracle binary in the reference's own
    shared-memory MPI mode: `ranks` ranks of one node (share_comm of all of
    them, SHN = ranks; the build's MPI shim forks them and lays the
    reference's shared windows in one arena), each marching its share of
    every array between the reference's own barriers.  Returns (rate, timed
    loop seconds, timed cell updates); the loop time is rank 0's between
    barriers that span every rank."""
    env = dict(os.environ, IB_STEPS=str(steps), IB_TIMED_FROM=str(warmup), IB_RANKS=str(ranks),
               IB_MPI_TIMEOUT=str(int(timeout)), **env_case)
    with tempfile.TemporaryDirectory() as wd:
        out = subprocess.run([binary], cwd=wd, env=env, stdout=subprocess.PIPE,
                             stderr=subprocess.DEVNULL, text=True, timeout=timeout + 120)
    if out.returncode != 0:
        raise RuntimeError(f"reference run failed (exit {out.returncode})")
    for line in out.stdout.splitlines():
        if line.startswith("ORACLE_RESULT"):
            r = json.loads(line.split(" ", 1)[1])
            if r.get("ranks", 1) != ranks:
                raise RuntimeError("reference run used another rank count")
            return r["cell_updates"] / r["loop_seconds"], r["loop_seconds"], r["cell_updates"]
    raise RuntimeError("reference run printed no result")


def reference_grid(n: int, ranks: int) -> int:
    """The largest n / 2^k grid whose reference run fits the host memory."""
    while n > 256 and (REF_SHARED_BYTES_2048 * (n / 2048) ** 2 + ranks * REF_RANK_BYTES
                       > 0.8 * avail_bytes()):
        n //= 2
    return n


def run_reference(n: int, steps: int, warmup: int = 0, ranks: int = 1):
    """The reference solver's own step (compiled from its sources) on the
    n x n vortex case in its shared-memory MPI mode with `ranks` ranks on the
    host cores.  Returns (cell_updates_per_s, seconds, cell_updates, kind, n)
    with n the grid run (smaller than asked only when the host memory is
    short).  Falls back to the C restatement on one core (kind "port") on a
    bounded grid when the reference build is absent."""
    binary = reference_binary()
    if binary is not None:
        n = reference_grid(n, ranks)
        rate, sec, upd = run_reference_mpi(binary, {"IB_NX": str(n), "IB_STAGES": str(STAGES)},
                                           steps, warmup, ranks)
        return rate, sec, upd, "reference", n
    n = min(n, PORT_SAMPLE_N)
    # C restatement of the same step
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import pyoracle
    pkg = load_pkg()
    P, cells, prim = pkg.workloads.vortex_case(n)
    d = dict(level=cells["level"], ix=cells["ix"], iy=cells["iy"],
             kind=np.zeros(n * n, np.int32), ptype=np.zeros(n * n, np.int32),
             solid=np.zeros(n * n, np.int32), infect=np.full(n * n, -1, np.int32),
             signdis=np.full(n * n, 9999.0), prim=prim.ravel(),
             dh=np.array(P["dh"][0]), schedule=np.array([1, 2, 2, 0, 1, 1], np.int32),
             domain=np.array([n, n, 1, 1, 0, 1], np.int32), initvar=np.array(P["initvar"]))
    gx, gy = [], []
    for y in range(-2, n + 2):
        for x in range(-2, n + 2):
            if x < 0 or y < 0 or x >= n or y >= n:
                gx.append(x)
                gy.append(y)
    gx, gy = np.array(gx, np.int32), np.array(gy, np.int32)
    for k, v in (("level", np.zeros_like(gx)), ("ix", gx), ("iy", gy), ("kind", np.full_like(gx, 2)),
                 ("ptype", np.zeros_like(gx)), ("solid", np.zeros_like(gx)),
                 ("infect", np.full_like(gx, -1)), ("signdis", np.full(len(gx), 9999.0))):
        d[k] = np.concatenate([d[k], v])
    d["prim"] = np.concatenate([prim, prim[(gy % n) * n + (gx % n)]]).ravel()
    lv = pyoracle.OracleLevels(d)
    dt = 1.0
    t0 = time.perf_counter()
    for ts in range(steps):
        if ts == warmup:
            t0 = time.perf_counter()
        rc, dt, _, _ = pyoracle.step(P, lv, ts, dt)
    sec = time.perf_counter() - t0
    upd = n * n * (steps - warmup)
    return upd / sec, sec, upd, "port", n


def reference_sample(kind: str, ranks: int, n: int, timed: int, warm: int) -> str:
    if kind == "port":
        return (f"the C restatement on one core, {timed} timed steps (after {warm}) of the same "
                f"case on a {n}x{n} grid")
    return (f"one run of the reference's own step in its shared-memory MPI mode: {ranks} ranks "
            f"(one per host core, SHN = {ranks}), {timed} timed steps (after {warm} warm-up) of "
            f"the {n}x{n} case; step loop only, between barriers over every rank")


def reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    ranks = host_cores() if reference_binary() else 1
    rate, sec, upd, kind, n = run_reference(args.n, args.warmup + args.steps, args.warmup, ranks)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3 / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"isentropic vortex {args.n}x{args.n} periodic, inviscid, "
                               "4-stage, VanLeer MUSCL, all-speed Roe, CFL 0.5",
                   "grid_run": f"{n}x{n}", "same_config": n == args.n and kind == "reference",
                   "parallelism": f"{ranks} MPI ranks of one shared-memory node"
                   if kind == "reference" else "one core"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": ranks, "kind": kind,
                         "sample": reference_sample(kind, ranks, n, args.steps, args.warmup)},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def lpt_shard(sizes, ws, rank):
    """Cases of this rank: greedy largest-first onto the least-loaded rank."""
    load = [0] * ws
    mine = []
    for i in sorted(range(len(sizes)), key=lambda k: -sizes[k]):
        r = min(range(ws), key=lambda k: load[k])
        load[r] += sizes[i]
        if r == rank:
            mine.append(i)
    return sorted(mine)


def batched_section(args, ib, wl, stream, barrier, max_over_ranks, ws, rank):
    """64 independent cases with uneven leaf counts, mixed precision, one
    persistent graph-replayed launch per stage (ibgpu_batch); cases sharded
    over the ranks (largest first), no data-path collective."""
    import torch
    cases = wl.batch_vortex_cases(BATCH_CASES, seed=0, precision=ib.MIXED)
    sizes = [len(c[1]["level"]) for c in cases]
    mine = lpt_shard(sizes, ws, rank)
    sols = []
    for i in mine:
        P, cells, prim = cases[i]
        s = ib.FlowSolver(P)
        s.set_stream(stream.cuda_stream)
        s.upload_topology(**cells)
        s.init_flow(prim)
        sols.append(s)
    del cases
    b = ib.Batch(sols)
    b.run(0, args.warmup)
    barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    b.run(args.warmup, args.steps)
    ev1.record(stream)
    ev1.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    barrier()
    b.set_timing(True)
    b.run(args.warmup + args.steps, min(args.steps, 5))
    info = b.info()
    total = sum(sizes)
    out = {"value": total * args.steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / args.steps,
           "cases": BATCH_CASES, "leaf_cells_total": total, "leaf_cells_min": min(sizes),
           "leaf_cells_max": max(sizes), "dtype": "f32 flux/limiter, f64 accumulation",
           "scaling": "strong", "sharding": "cases, largest first, no collective",
           "persistent_ctas": info["grid"], "block_threads": info["threads"],
           "autotune_ms": info["tuning"],
           "stage_ms_per_launch": info["stage_ms"] / max(info["stage_launches"], 1),
           "workload": "periodic vortex cases, side 16k with n^2 log-uniform in [5e4, 8e5], "
                       "Mach U[0.1,0.8], direction U[-5,10] deg (seed 0), single level"}
    b.close()
    return out, sols, [sizes[i] for i in mine]


def learned_section(ib, wl, ind, sols, sizes, stream, batched_ms_per_step):
    """Learned refinement indicator: trained on the GPU from the plain
    criterion's tags of the NACA0012 record, held-out mismatch, and the cost
    of learned tagging of every leaf box of the batched cases once per
    regrid added to the batched step time."""
    import numpy as np
    import torch
    rec = np.load(NACA_RECORD)
    g = {k: rec[k] for k in rec.files}
    sol = wl.naca_solver(g, 0, ib.FP64)
    sol.set_stream(stream.cuda_stream)
    t = g["tags"]
    key = t[:, 0] * 1e8 + t[:, 1] * 1e4 + t[:, 2]
    _, first = np.unique(key, return_index=True)
    t = t[np.sort(first)]
    mesh = set(zip(g["level"].tolist(), g["ix"].tolist(), g["iy"].tolist()))
    t = t[[(int(a), int(b), int(c)) in mesh for a, b, c in t[:, :3]]]
    B = dict(level=t[:, 0].astype(np.int32), ix=t[:, 1].astype(np.int32), iy=t[:, 2].astype(np.int32),
             xc=t[:, 3], yc=t[:, 4], signdis=t[:, 5])
    dh = g["dh"].reshape(-1, 3)[:, 0]
    rule = wl.naca_tag_rule(int(g["domain"][5]), dh)
    labels = ind.classes_from_tags(sol.tag_plain(rule, B["level"], B["xc"], B["yc"], B["signdis"]))
    li = ind.LearnedIndicator(sol, seed=0)
    feats = []
    for s in range(4):
        feats.append(li.features(rule, B))
        sol.run(2 * s, 2)
    n = len(labels)
    hold = np.random.default_rng(0).random(n) < 0.2
    keep = torch.from_numpy(~hold).cuda()
    Xtr = torch.cat([f[keep] for f in feats[:-1]]).contiguous()
    ytr = np.concatenate([labels[~hold]] * 3)
    Xte = feats[-1][torch.from_numpy(hold).cuda()].contiguous()
    yte = labels[hold]
    untrained = float(np.mean(li.predict(Xte) != yte))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    steps = 600
    li.train(Xtr, ytr, steps=steps, batch=4096, lr=3e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    trained = float(np.mean(li.predict(Xte) != yte))
    majority = float(np.mean(yte != np.bincount(ytr, minlength=3).argmax()))
    # learned tagging of every leaf box of this rank's batched cases, from
    # the device state (features gathered inside the tensor-core kernel), and
    # the plain criterion over the same boxes for comparison
    boxes = sum(s.ncells for s in sols)
    tb = ib.Batch(sols) if sols else None
    reps = {0: [], 1: []}
    with near_gpu_cores(torch.cuda.current_device()):
        tags_host = torch.empty(max(boxes, 1), dtype=torch.uint8).pin_memory().numpy()
        for learned in (1, 0):
            dp = li.params.data_ptr() if learned else 0
            if tb:
                tb.tag_mesh(rule, dp, tags_host)  # warm-up (kernel attributes)
            for _ in range(3):  # best of three passes over all cases (host noise)
                torch.cuda.synchronize()
                t1 = time.perf_counter()
                if tb:
                    tb.tag_mesh(rule, dp, tags_host)
                reps[learned].append((time.perf_counter() - t1) * 1e3)
    if tb:
        tb.close()
    tag_ms, plain_ms = min(reps[1]), min(reps[0])
    sol.close()
    per_step = batched_ms_per_step + tag_ms / REGRID_EVERY
    return {"tag_mismatch_heldout": trained, "tag_mismatch_untrained": untrained,
            "tag_mismatch_majority_class": majority, "train_steps": steps,
            "train_rows_per_s": steps * 4096 / train_s,
            "tag_boxes_per_s": boxes / (tag_ms / 1e3) if tag_ms > 0 else None,
            "tag_ms_all_boxes": tag_ms, "plain_tag_ms_all_boxes": plain_ms,
            "regrid_every": REGRID_EVERY,
            "gain_over_plain": "none measured: the labels are the plain criterion's decisions, "
                               "which it reproduces (held-out mismatch above) at "
                               f"{tag_ms / max(plain_ms, 1e-9):.1f}x the plain criterion's "
                               "tagging time; learned regrids of the reference's NACA0012 run "
                               "move the level-1 leaf count from 3944 to about 4170 and Cl/Cd "
                               "by up to 5.8e-4 (tests/test_gpu_learned_regrid.py)",
            "value": sum(sizes) / (per_step / 1e3), "unit": UNIT,
            "value_note": "batched mixed solver with learned tagging of every leaf box once per "
                          "regrid (ibgpu_batch_tag_mesh wall time incl. the tags' copy-back into "
                          "pinned memory, amortised over the regrid interval)",
            "cl_cd_deviation": None,
            "cl_cd_note": "the regrid is the reference's host code: measured by "
                          "tests/test_gpu_learned_regrid.py (the reference's NACA0012 run "
                          "regridding every 2 steps on this indicator's GPU decisions, 400 "
                          "steps): max |dCd| 2.1e-4, max |dCl| 5.8e-4 vs the plain criterion"}


def load_record(path):
    import numpy as np
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def marched_cells(g, ts0: int, nsteps: int) -> int:
    """Leaf-cell updates of steps ts0 .. ts0+nsteps-1 of a record's mesh: the
    normal cells of the levels that march each step (subcycling schedule)."""
    import numpy as np
    sched = g["schedule"].reshape(-1, 6)
    per_level = np.bincount(g["level"][g["kind"] == 0], minlength=len(sched))
    return int(sum(per_level[l] for ts in range(ts0, ts0 + nsteps) for l in range(len(sched))
                   if ts % sched[l, 0] == sched[l, 3]))


def config1_section(ib, wl, stream, max_over_ranks, timed_steps: int = 400, rank: int = 0):
    """The plain-method airfoil workload at its stated size (the reference's
    mesh and initial state): FP64 and mixed leaf-cell updates/s (levels that
    march only), |dCl|, |dCd| of both over the 1000 steps against the
    reference's own history, and the reference's step on the same case on
    the host cores."""
    import numpy as np
    import torch
    g = load_record(CONFIG1_RECORD)
    hist = load_record(CONFIG1_HISTORY)["history"]
    period = int(g["schedule"].reshape(-1, 6)[:, 0].max())  # one coarse-level period
    out = {"workload": "static NACA0012 (400 surface points) on a 128x128 base grid of "
                       "[0,20]^2 + 3 AMR levels, Mach 0.5, 2 deg, Re 5000, minmod, 4-stage, "
                       "CFL 0.5; the reference's own mesh and initial state",
           "leaf_cells": int((g["kind"] == 0).sum()),
           "cell_updates_per_step": marched_cells(g, 0, period) / period}
    cl_cd = lambda f: np.asarray(f).reshape(-1, 6)[:, :2].sum(axis=0) / F_REF  # noqa: E731
    ends = {}
    for name, prec in (("fp64", ib.FP64), ("mixed", ib.MIXED)):
        s = wl.naca_solver(g, 0, prec)
        s.set_stream(stream.cuda_stream)
        s.run(0, period)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        s.run(period, timed_steps)
        ev1.record(stream)
        ev1.synchronize()
        ms = max_over_ranks(ev0.elapsed_time(ev1))
        s.close()
        upd = marched_cells(g, period, timed_steps)
        # the same case through the batch entry point with one case: each
        # step one CUDA graph replay, the stage launches merged over levels
        s = wl.naca_solver(g, 0, prec)
        s.set_stream(stream.cuda_stream)
        b = ib.Batch([s])
        b.run(0, 2 * period)
        torch.cuda.synchronize()
        ev0.record(stream)
        b.run(2 * period, timed_steps)
        ev1.record(stream)
        ev1.synchronize()
        ms_graph = max_over_ranks(ev0.elapsed_time(ev1))
        info = b.info()
        b.close()
        s.close()
        upd_graph = marched_cells(g, 2 * period, timed_steps)
        # accuracy: the stated 1000 steps from the initial state, forces each step
        s = wl.naca_solver(g, 0, prec)
        s.set_stream(stream.cuda_stream)
        worst = np.zeros(2)
        for k in range(len(hist)):
            s.time_marching(k)
            f = s.wall_forces()
            worst = np.maximum(worst, np.abs(cl_cd(f) - cl_cd(hist[k, 3:])))
        ends[name] = cl_cd(s.wall_forces())
        s.close()
        out[name] = {"value": upd / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / timed_steps,
                     "timed_steps": timed_steps,
                     "max_dcd_vs_reference": float(worst[0]), "max_dcl_vs_reference": float(worst[1]),
                     "graph": {"value": upd_graph / (ms_graph / 1e3), "unit": UNIT,
                               "ms_per_step": ms_graph / timed_steps,
                               "path": "ibgpu_batch_run of this one case (CUDA graph per step)",
                               "persistent_ctas": info["grid"],
                               "block_threads": info["threads"]}}
    out["cd_cl_reference_step1000"] = cl_cd(hist[-1, 3:]).tolist()
    out["mixed_vs_fp64_step1000"] = np.abs(ends["mixed"] - ends["fp64"]).tolist()
    out["gate_1e-3"] = bool(max(out["mixed"]["max_dcd_vs_reference"],
                                out["mixed"]["max_dcl_vs_reference"]) < 1e-3)
    out["cl_cd_note"] = ("Cd, Cl = x, y force of both surfaces over 0.5 rho u^2 c dz; max over "
                         "every step of the 1000-step run against the reference's own history")
    binary = os.path.join(ROOT, "oracle", "_ref", "ref_naca_minmod")
    if rank == 0 and os.path.exists(binary):
        ranks = host_cores()
        rate, sec, upd = run_reference_mpi(binary, CONFIG1_ENV, 5 * period, period, ranks)
        out["reference"] = {"value": rate, "unit": UNIT, "cores": ranks,
                            "sample": f"the reference's own step on this case in its "
                                      f"shared-memory MPI mode, {ranks} ranks (one per host "
                                      f"core), {4 * period} timed steps after {period}"}
    return out


def run_oracle_binary(binary: str, env_case: dict, extra: dict, timeout: float = 900.0):
    """One reference-solver process (its ORACLE_RESULT line and force log)."""
    import numpy as np
    with tempfile.TemporaryDirectory() as wd:
        log = os.path.join(wd, "forces.bin")
        env = dict(os.environ)
        env.update(env_case)
        env.update(extra)
        env["IB_FORCE_LOG"] = log
        out = subprocess.run([binary], cwd=wd, env=env, capture_output=True, text=True,
                             timeout=timeout)
        if out.returncode != 0:
            raise RuntimeError(f"{os.path.basename(binary)} failed: {out.stderr[-500:]}")
        res = next(json.loads(l.split(" ", 1)[1]) for l in out.stdout.splitlines()
                   if l.startswith("ORACLE_RESULT"))
        hist = np.fromfile(log, np.float64)
    steps = int(env_case.get("IB_STEPS", extra.get("IB_STEPS", 0)))
    return res, hist.reshape(steps, -1) if steps else hist


def config3_section(steps: int = 42, warm: int = 2, rank: int = 0):
    """The moving-body workload at its stated size, stepped by the
    reference's own main loop through the C++ binding (GpuNS_Solver) in the
    reference's shared-memory MPI mode on the host cores: every step all
    ranks move and re-immerse the body with the reference's code over their
    shares of the mesh, rank 0 hands the device the new flags and
    immersed-boundary records and the device runs the step.  FP64 and mixed
    runs: leaf-cell updates/s of the device step alone and of the whole step
    including the host's re-immersion (40 timed steps from step 2, so two of
    the workload's regrids, at steps 20 and 40, fall inside them and their
    cost is spread over the steps), the host time per step, and |dCl|,
    |dCd| of mixed against FP64; the reference's own step (motion included)
    on the same mesh and ranks, run after the GPU runs."""
    import numpy as np
    binding = os.path.join(ROOT, "oracle", "_ref", "ref_pitch_minmod_binding")
    if rank != 0 or not os.path.exists(binding):
        return None
    out = {"workload": "NACA0015 pitching about the quarter chord (5 deg, k 0.1, mean 0), Mach "
                       "0.2, Re 1e4, 256x256 base grid on [0,30]^2 + 5 AMR levels tracking the "
                       "body and wake, regrid every 20 steps; mesh, motion and re-immersion by "
                       "the reference's own host code",
           "timed_steps": steps - warm,
           "regrids_timed": len([t for t in range(warm, steps) if t > 0 and t % 20 == 0])}
    # regrid_ms_each: one regrid's time; regrid_phases_s_total: its parts
    # summed over the timed regrids
    nreg = max(out["regrids_timed"], 1)
    hist = {}
    ranks = host_cores()
    for name, prec in (("fp64", 0), ("mixed", 2)):
        res, h = run_oracle_binary(binding, CONFIG3_ENV,
                                   {"IB_STEPS": str(steps), "IB_TIMED_FROM": str(warm),
                                    "IB_BINDING_STEP": "1", "IB_BINDING_PRECISION": str(prec),
                                    "IB_RANKS": str(ranks), "IB_MPI_TIMEOUT": "900"})
        hist[name] = h
        dev_s = res["loop_seconds"] - res["move_seconds"]
        out[name] = {"value": res["cell_updates"] / dev_s, "unit": UNIT,
                     "device_ms_per_step": dev_s * 1e3 / (steps - warm),
                     "with_host_reimmersion": res["cell_updates"] / res["loop_seconds"],
                     "host_reimmersion_ms_per_step": res["move_seconds"] * 1e3 / (steps - warm),
                     "regrid_ms_each": res.get("regrid_seconds", 0.0) * 1e3 / nreg,
                     "regrid_phases_s_total": res.get("regrid_phases_seconds"),
                     "with_regrids": res["cell_updates"] / (res["loop_seconds"] +
                                                            res.get("regrid_seconds", 0.0)),
                     "host_ranks": res.get("ranks", 1),
                     "host_phases_s_all_steps": res.get("move_phases_seconds"),
                     "cell_updates_per_step": res["cell_updates"] / (steps - warm)}
    f = {k: v[:, 3:].reshape(len(v), -1, 6)[:, :, :2].sum(axis=1) / F_REF for k, v in hist.items()}
    d = np.abs(f["mixed"] - f["fp64"]).max(axis=0)
    out["mixed_vs_fp64_max_dcd"], out["mixed_vs_fp64_max_dcl"] = float(d[0]), float(d[1])
    out["device_step_note"] = ("device step = the synchronous ibgpu_step wall time (loop time "
                               "minus the host's motion, re-immersion and record upload); the "
                               f"host part runs on {ranks} MPI ranks of the reference, rank 0 "
                               "driving the device; with_host_reimmersion counts the timed "
                               "steps (the first step after a regrid packs every wall pair); "
                               "with_regrids adds the regrid between them (tagging, the "
                               "reference's PerformAdaptive, download and upload)")
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_pitch_minmod")
    if os.path.exists(ref):
        ranks = host_cores()
        # the same window as the GPU runs: 20 timed steps from step 2, the
        # regrid at step 20 between them
        res, _ = run_oracle_binary(ref, CONFIG3_ENV,
                                   {"IB_STEPS": str(steps), "IB_TIMED_FROM": str(warm),
                                    "IB_RANKS": str(ranks), "IB_MPI_TIMEOUT": "900"},
                                   timeout=1800.0)
        if res.get("ranks", 1) != ranks:
            raise RuntimeError("reference run used another rank count")
        out["reference"] = {"value": res["cell_updates"] / res["loop_seconds"], "unit": UNIT,
                            "cores": ranks,
                            "regrid_ms_each": res.get("regrid_seconds", 0.0) * 1e3 / nreg,
                            "regrid_phases_s_total": res.get("regrid_phases_seconds"),
                            "with_regrids": res["cell_updates"] / (
                                res["loop_seconds"] + res.get("regrid_seconds", 0.0)),
                            "sample": f"the reference's own step with its moving-body path in "
                                      f"its shared-memory MPI mode, {ranks} ranks (one per host "
                                      f"core), {steps - warm} timed steps after {warm} (the "
                                      f"regrids at steps 20 and 40 timed apart, as for the GPU "
                                      f"runs)"}
    return out


def config4_cases(ncases: int = CONFIG4_CASES, seed: int = 0):
    """The batched airfoil cases: per case, in this order from one seeded
    generator, Mach U[0.1, 0.8], angle of attack U[-5, 10] deg, Re
    log-uniform in [2e3, 2e4], AMR levels U{2..5} above the base grid (3..6
    mesh levels, as the plain-method workload's "128^2 plus 3 AMR levels" is
    4) and a target leaf count log-uniform in [5e4, 8e5] that sets the base
    grid; profile NACA0012 and NACA0015 alternating.  Returns the reference
    case environments."""
    import math
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for i in range(ncases):
        mach = float(rng.uniform(0.1, 0.8))
        aoa = float(rng.uniform(-5.0, 10.0))
        re = math.exp(float(rng.uniform(math.log(2e3), math.log(2e4))))
        levels = int(rng.integers(2, 6)) + 1  # mesh levels: the base grid and 2..5 AMR levels
        target = math.exp(float(rng.uniform(math.log(5e4), math.log(8e5))))
        nx = max(64, int(round(math.sqrt(target / CONFIG4_LEAF_FACTOR[levels]) / 16.0)) * 16)
        out.append({"IB_MACH": repr(mach), "IB_AOA": repr(aoa), "IB_RE": repr(re),
                    "IB_LEVELS": str(levels), "IB_NX": str(nx),
                    "IB_THICK": "0.12" if i % 2 == 0 else "0.15", "IB_NPTS": "200",
                    "IB_STAGES": "4", "IB_USER_INIT": "0", "IB_STEPS": "0"})
    return out


def config4_meshes(envs, workers: int):
    """The cases' meshes and initial states from the reference's own mesh
    generation (one process per case, `workers` at a time), as records."""
    from concurrent.futures import ThreadPoolExecutor
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden
    import pyoracle
    binary = os.path.join(ROOT, "oracle", "_ref", "ref_naca_minmod")

    def one(env_case):
        with tempfile.TemporaryDirectory() as wd:
            env = dict(os.environ)
            env.update(env_case)
            env["IB_DUMP"] = os.path.join(wd, "d")
            subprocess.run([binary], cwd=wd, env=env, check=True, stdout=subprocess.DEVNULL,
                           stderr=subprocess.DEVNULL, timeout=900)
            return make_golden.record_of(pyoracle.read_dump(os.path.join(wd, "d_000000.bin")))

    with ThreadPoolExecutor(max(1, workers)) as pool:
        return list(pool.map(one, envs))


def config4_section(ib, wl, ind, stream, ncases: int, steps: int, warm: int = 4):
    """The batched airfoil workload: ncases of the seeded 64 (the reference's
    own meshes, 2-5 levels, an immersed airfoil each) in one batch, mixed
    precision and FP64, persistent graph-replayed stage launches; leaf-cell
    updates/s over the levels that march; |dCl|, |dCd| of mixed against FP64
    per case after the run; tagging of every leaf box by the learned
    indicator and by the plain criterion."""
    import numpy as np
    import torch
    envs = config4_cases()[:ncases]
    t0 = time.perf_counter()
    recs = config4_meshes(envs, host_workers(1.5e9))
    mesh_s = time.perf_counter() - t0
    leaves = [int((g["kind"] == 0).sum()) for g in recs]
    per_step = sum(marched_cells(g, warm, steps) for g in recs) / steps
    out = {"workload": f"the first {ncases} of 64 seeded NACA0012/0015 cases (seed 0): Mach "
                       "U[0.1,0.8], AoA U[-5,10] deg, Re log-U[2e3,2e4], 2-5 AMR levels, "
                       "leaf-count target log-U[5e4,8e5]; meshes and initial states from the "
                       "reference's own mesh generation",
           "cases": ncases, "leaf_cells_total": sum(leaves), "leaf_cells_min": min(leaves),
           "leaf_cells_max": max(leaves), "cell_updates_per_step": per_step,
           "host_mesh_generation_s": mesh_s, "timed_steps": steps}
    forces = {}
    for name, prec in (("mixed", ib.MIXED), ("fp64", ib.FP64)):
        sols = []
        for g in recs:
            s = wl.naca_solver(g, 0, prec)
            s.set_stream(stream.cuda_stream)
            sols.append(s)
        b = ib.Batch(sols)
        b.run(0, warm)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        b.run(warm, steps)
        ev1.record(stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
        info = b.info()
        out[name] = {"value": per_step * steps / (ms / 1e3), "unit": UNIT,
                     "ms_per_step": ms / steps, "persistent_ctas": info["grid"],
                     "block_threads": info["threads"]}
        forces[name] = [s.wall_forces()[:, :2].sum(axis=0) / F_REF for s in sols]
        if name == "mixed":
            # tagging of every box of every case: learned (an untrained
            # network costs what a trained one does) and plain
            li = ind.LearnedIndicator(sols[0], seed=0)
            rule = wl.naca_tag_rule(5, [20.0 / 128 / 2 ** k for k in range(5)])
            nbox = sum(s.ncells for s in sols)
            tags = torch.empty(nbox, dtype=torch.uint8).pin_memory().numpy()
            for learned, key in ((1, "learned_tag_ms"), (0, "plain_tag_ms")):
                dp = li.params.data_ptr() if learned else 0
                b.tag_mesh(rule, dp, tags)
                best = []
                for _ in range(3):
                    torch.cuda.synchronize()
                    t1 = time.perf_counter()
                    b.tag_mesh(rule, dp, tags)
                    best.append((time.perf_counter() - t1) * 1e3)
                out[key] = min(best)
            out["tag_boxes"] = nbox
            out["learned_value"] = per_step / ((ms / steps + out["learned_tag_ms"] / REGRID_EVERY)
                                               / 1e3)
        b.close()
        for s in sols:
            s.close()
    d = np.abs(np.array(forces["mixed"]) - np.array(forces["fp64"]))
    out["mixed_vs_fp64_max_dcd"], out["mixed_vs_fp64_max_dcl"] = float(d[:, 0].max()), float(d[:, 1].max())
    out["gate_1e-3"] = bool(d.max() < 1e-3)
    out["learned_note"] = ("learned_value: the mixed batch with learned tagging of every leaf box "
                           f"once per {REGRID_EVERY} steps; the regrid itself is the reference's "
                           "host code and not timed")
    return out


def accuracy_section(ib, wl, stream, n: int = 2048, steps: int = 500):
    """The bandwidth workload's accuracy: the 2048^2 vortex after `steps`
    steps, L2 density error vs the exact solution for FP64 and mixed, and
    mixed vs FP64 (the airfoil gate is in the config1 section)."""
    import numpy as np
    out = {}
    dens = {}
    tfin = {}
    for name, prec in (("fp64", ib.FP64), ("mixed", ib.MIXED)):
        P, cells, prim = wl.vortex_case(n, precision=prec)
        s = ib.FlowSolver(P)
        s.set_stream(stream.cuda_stream)
        s.upload_topology(**cells)
        s.init_flow(prim)
        t = 0.0
        for ts in range(steps):
            s.time_marching(ts)
            t += s.dt  # the dt this step used
        dens[name] = s.download()[:, 0]
        tfin[name] = t
        s.close()
    out["vortex_steps"] = steps
    rho_fp64, rho_mixed = dens["fp64"], dens["mixed"]
    for name in ("fp64", "mixed"):
        exact = wl.vortex_exact_density(n, tfin[name])
        out[f"vortex_l2_rho_{name}_vs_exact"] = float(np.sqrt(np.mean((dens[name] - exact) ** 2)))
    out["vortex_l2_rho_mixed_vs_fp64"] = float(np.sqrt(np.mean((rho_mixed - rho_fp64) ** 2)))
    return out


def our_arm(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    pkg = load_pkg()
    ib, wl = pkg.ibgpu, pkg.workloads
    n = args.n
    ncell = n * n

    stream = torch.cuda.Stream(device=dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if ws > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def make(precision):
        P, cells, prim = wl.vortex_case(n, nstages=STAGES, precision=precision)
        sol = ib.FlowSolver(P)
        sol.set_stream(stream.cuda_stream)
        sol.upload_topology(**cells)
        sol.init_flow(prim)
        return sol, prim

    def timed_steps(sol, first_ts, k, sampler=None):
        barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        if sampler:
            sampler.start()
        ev0.record(stream)
        sol.run(first_ts, k)  # k steps back to back, dt kept on the device
        ev1.record(stream)
        ev1.synchronize()
        clocks = sampler.stop() if sampler else None
        barrier()
        return ev0.elapsed_time(ev1), clocks

    # ---- FP64 plain path (headline)
    sol, prim = make(ib.FP64)
    sol.run(0, args.warmup)
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    ms, clocks, remeasured = timed_with_retry(
        lambda: timed_steps(sol, args.warmup, args.steps, sampler), max_over_ranks)
    if clocks is not None:
        clocks = dict(clocks, remeasured=remeasured)
    ms = max_over_ranks(ms)
    value = ncell * args.steps * ws / (ms / 1e3)

    # stage-kernel duration (CUDA events on the launching stream)
    sol.set_kernel_timing(True)
    kt_steps = min(args.steps, 10)
    sol.run(args.warmup + args.steps, kt_steps)
    kms, kn = sol.kernel_times()
    sol.set_kernel_timing(False)
    stage_ms = kms[0] / max(kn[0], 1)
    stage_bytes = BYTES_PER_CELL_STAGE * ncell
    achieved = stage_bytes / (stage_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profile_traffic()

    # ---- e2e through the C ABI with pinned host buffers: every step uploads
    # the state, steps, and reads the state back, all enqueued without host
    # waits (ibgpu_upload_state_async / ibgpu_step_async /
    # ibgpu_download_state_async, one ibgpu_step_result at the end): the
    # upload and read-back run on their own streams, so the copies of one
    # step overlap each other (PCIe is full duplex) and the neighbouring
    # steps' compute; all of it is inside the timed region
    # compact rows (roe, u, v, p): T and e follow from them on upload
    # the same K steps as the device-timed line (the pipeline's fill and
    # drain, one upload and one read-back not overlapped, are in the region)
    e2e_steps = max(3, args.steps)
    sol.set_state_rows(ib.ROWS_COMPACT)
    with near_gpu_cores(torch.cuda.current_device()) as e2e_cores:
        host_in = torch.from_numpy(np.ascontiguousarray(prim[:, [0, 1, 2, 4]])).pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        # warm-up of the pipelined path (untimed), as for the device-timed line
        for s in range(2):
            sol.upload_async(host_in.data_ptr())
            sol.step_async(s)
            sol.download_async(host_out.data_ptr())
        sol.step_result()
        sol.synchronize()
        barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        t0 = time.perf_counter()
        for s in range(e2e_steps):
            sol.upload_async(host_in.data_ptr())
            sol.step_async(s)
            sol.download_async(host_out.data_ptr())
        sol.step_result()
        sol.synchronize()
        ev1.record(stream)
        ev1.synchronize()
        # the transfer bound of this path: the same bytes each way at once,
        # plain copies on two streams, no compute
        dev_a = torch.empty_like(host_in, device="cuda")
        dev_b = torch.empty_like(host_in, device="cuda")
        s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
        torch.cuda.synchronize()
        b0 = torch.cuda.Event(enable_timing=True)
        b1 = torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        for _ in range(3):
            s_in.wait_stream(stream)
            s_out.wait_stream(stream)
            with torch.cuda.stream(s_in):
                dev_a.copy_(host_in, non_blocking=True)
            with torch.cuda.stream(s_out):
                host_out.copy_(dev_b, non_blocking=True)
            stream.wait_stream(s_in)
            stream.wait_stream(s_out)
        b1.record(stream)
        b1.synchronize()
        duplex_ms = b0.elapsed_time(b1) / 3
        del dev_a, dev_b
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1))
    e2e_value = ncell * e2e_steps * ws / (e2e_ms / 1e3)
    sol.close()

    # ---- mixed precision (FP32 flux/limiter, FP64 accumulation)
    msol, _ = make(ib.MIXED)
    msol.run(0, args.warmup)
    mms, _ = timed_steps(msol, args.warmup, args.steps)
    mms = max_over_ranks(mms)
    mixed_value = ncell * args.steps * ws / (mms / 1e3)
    msol.set_kernel_timing(True)
    msol.run(args.warmup + args.steps, kt_steps)
    mk, mkn = msol.kernel_times()
    msol.close()

    # ---- batched cases, learned indicator, accuracy reports
    extra = {}
    if not args.headline_only:
        bat, bsols, bsizes = batched_section(args, ib, wl, stream, barrier, max_over_ranks, ws, rank)
        extra["batched"] = bat
        extra["learned"] = learned_section(ib, wl, pkg.indicator, bsols, bsizes, stream,
                                           bat["ms_per_step"])
        for s in bsols:
            s.close()
        extra["config1"] = config1_section(ib, wl, stream, max_over_ranks, rank=rank)
        if rank == 0 and args.config4_cases > 0:
            extra["config4"] = config4_section(ib, wl, pkg.indicator, stream, args.config4_cases,
                                               steps=args.steps)
        if not args.no_config3:
            extra["config3"] = config3_section(rank=rank)
        if rank == 0:
            extra["accuracy"] = accuracy_section(ib, wl, stream, n=n)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        ranks = host_cores() if reference_binary() else 1
        rate, sec, upd, kind, rn = run_reference(n, 4, 1, ranks)
        cpu = {"value": rate, "unit": UNIT, "cores": ranks, "kind": kind,
               "sample": reference_sample(kind, ranks, rn, 3, 1) + f"; {upd} timed leaf-cell "
                         "updates"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"isentropic vortex {n}x{n} periodic on [0,10]^2, strength 5, "
                                   "Mach 0.5 at 45 deg, inviscid, 4-stage low-storage scheme, "
                                   "VanLeer MUSCL, all-speed Roe, CFL 0.5",
                       "leaf_cells": ncell, "precision": "fp64",
                       "l2": "state (~470 MB incl. stage buffers) larger than L2; no flush",
                       "parallelism": "replicas" if ws > 1 else "single GPU"},
            # one timed run of K steps: the first step launches the CFL pass
            # and dt finalisation, later steps the reduction reset and the
            # take-over of the CFL bound folded into the previous final
            # stage; every step one launch per stage
            "gpu_launches": (2 + STAGES) * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "stage_kernel (flux + residual + update + prim recovery)",
                         "bytes_per_launch": stage_bytes, "ms_per_launch": stage_ms,
                         "peak_source": peak_kind},
            "e2e": {"value": e2e_value, "unit": UNIT, "steps": e2e_steps,
                    "ms_per_step": e2e_ms / e2e_steps,
                    "transfer_bound_ms_per_step": duplex_ms,
                    "frac_of_transfer_bound": duplex_ms / (e2e_ms / e2e_steps),
                    "h2d_bytes_per_step": ncell * 4 * 8,
                    "d2h_bytes_per_step": ncell * 4 * 8,
                    "path": "compact rows (roe, u, v, p; ibgpu_set_state_rows): "
                            "ibgpu_upload_state_async + ibgpu_step_async + "
                            "ibgpu_download_state_async per step, ibgpu_step_result and "
                            "ibgpu_synchronize at the end",
                    "host_cores": (f"{len(e2e_cores)} cores of the GPU's NUMA node (pinned "
                                   "buffers allocated there)") if e2e_cores else "unbound"},
            "mixed": {"value": mixed_value, "unit": UNIT, "ms_per_step": mms / args.steps,
                      "stage_ms_per_launch": mk[0] / max(mkn[0], 1),
                      # same algorithmic bytes per launch as the FP64 line (U^n
                      # and U^(k) stay FP64 in the definition)
                      "roofline_frac": (stage_bytes / (mk[0] / max(mkn[0], 1) / 1e3) / 1e9) / peak
                      if peak and mk[0] > 0 else None,
                      "dtype": "f32 flux/limiter, f64 accumulation"},
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def profile_run(args):
    """A short run of one workload on cuda:0, as the command under ncu:
      stage     --n N --steps K --precision P  the periodic vortex, K full
                steps after one (kernel of interest: stage_kernel)
      batch     --cases C --grid G --precision P  C batched vortex cases
                (50k..800k cells, seed 0)
      mlp-grad  --rows R --steps K  K learned-indicator training steps on R
                random BF16 rows (mlp_grad_kernel)
      mlp-tag   --n N --steps K  learned tagging of every cell of an N x N
                vortex case (mlp_tag_mesh_kernel)
    Prints the mean wall time per step; no JSON line."""
    import numpy as np
    import torch
    pkg = load_pkg()
    ib, wl, ind = pkg.ibgpu, pkg.workloads, pkg.indicator
    prec = {"fp64": ib.FP64, "exact": ib.FP64_EXACT, "mixed": ib.MIXED}[args.precision]
    k = max(args.steps, 1)
    if args.profile == "stage":
        P, cells, prim = wl.vortex_case(args.n, precision=prec)
        sol = ib.FlowSolver(P)
        sol.upload_topology(**cells)
        sol.init_flow(prim)
        sol.time_marching(0)
        t0 = time.perf_counter()
        sol.run(1, k)
        dt = (time.perf_counter() - t0) / k
        print(f"{args.n}x{args.n} {args.precision}: {dt * 1e3:.3f} ms/step (wall, {k} steps)")
        sol.close()
    elif args.profile == "batch":
        sols = []
        for P, cells, prim in wl.batch_vortex_cases(args.cases, seed=0, precision=prec):
            s = ib.FlowSolver(P)
            s.upload_topology(**cells)
            s.init_flow(prim)
            sols.append(s)
        b = ib.Batch(sols)
        b.set_grid(args.grid)
        b.run(0, 1)
        t0 = time.perf_counter()
        b.run(1, k)
        dt = (time.perf_counter() - t0) / k
        ncell = sum(s.ncells for s in sols)
        print(f"batch of {args.cases} cases ({ncell} cells) {args.precision}: {dt * 1e3:.3f} "
              f"ms/step (wall), {b.info()}")
        b.close()
        for s in sols:
            s.close()
    elif args.profile == "mlp-grad":
        P, cells, prim = wl.vortex_case(64)
        sol = ib.FlowSolver(P)
        rng = np.random.default_rng(0)
        X = rng.normal(0, 1, (args.rows, ib.MLP_IN)).astype(np.float32)
        feat = torch.from_numpy((X.view(np.uint32) >> 16).astype(np.uint16).view(np.int16)).cuda()
        y = rng.integers(0, 3, args.rows).astype(np.uint8)
        li = ind.LearnedIndicator(sol, seed=0)
        li.train(feat, y, steps=2, batch=args.rows)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        li.train(feat, y, steps=k, batch=args.rows)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / k
        print(f"{args.rows} rows: {dt * 1e3:.3f} ms per training step (wall)")
        sol.close()
    else:  # mlp-tag
        P, cells, prim = wl.vortex_case(args.n)
        sol = ib.FlowSolver(P)
        sol.upload_topology(**cells)
        sol.init_flow(prim)
        li = ind.LearnedIndicator(sol, seed=0)
        rule = wl.naca_tag_rule(1, [10.0 / args.n])
        sol.tag_mesh(rule, li.params.data_ptr())
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k):
            tags = sol.tag_mesh(rule, li.params.data_ptr())
        dt = (time.perf_counter() - t0) / k
        print(f"{args.n}x{args.n}: {dt * 1e3:.3f} ms per ibgpu_tag_mesh call, tag counts "
              f"{np.bincount(tags, minlength=4).tolist()}")
        sol.close()
    return 0


def spawn_ranks(n: int, cmd: list, extra_env: dict | None = None, timeout: float = 3600.0):
    """Run cmd as n ranks of one job on this node (RANK, LOCAL_RANK,
    WORLD_SIZE, MASTER_ADDR/PORT set per process, 127.0.0.1 rendezvous);
    the ranks share this process's stdout.  Returns the exit codes; every
    rank is stopped when one fails or the time runs out."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n),
                   LOCAL_WORLD_SIZE=str(n), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                   **(extra_env or {}))
        procs.append(subprocess.Popen(cmd, env=env))
    deadline = time.monotonic() + timeout
    codes = [None] * n
    while any(c is None for c in codes):
        for i, p in enumerate(procs):
            if codes[i] is None:
                codes[i] = p.poll()
        if any(c not in (None, 0) for c in codes) or time.monotonic() > deadline:
            for i, p in enumerate(procs):
                if codes[i] is None:
                    p.kill()
                    codes[i] = p.wait()
            break
        time.sleep(0.05)
    return codes


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config4-cases", type=int, default=CONFIG4_DEFAULT_CASES,
                    help="batched airfoil cases of the seeded 64 to run (0 skips the section)")
    ap.add_argument("--no-config3", action="store_true",
                    help="skip the moving-body section (about three minutes of host mesh work)")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the batched, learned-indicator, airfoil and accuracy sections")
    ap.add_argument("--profile", choices=["stage", "batch", "mlp-grad", "mlp-tag"],
                    help="instead of the benchmark: a short run of one workload as the command "
                         "under a profiler (see profile_run)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "exact", "mixed"])
    ap.add_argument("--cases", type=int, default=16, help="--profile batch: batched cases")
    ap.add_argument("--grid", type=int, default=-1,
                    help="--profile batch: CTA count of the merged launches (0 one per item, "
                         "-1 autotuned)")
    ap.add_argument("--rows", type=int, default=262144, help="--profile mlp-grad: rows")
    args = ap.parse_args(argv)
    if args.profile:
        return profile_run(args)
    if args.warmup < 3:
        args.warmup = 3
    ws_env = os.environ.get("WORLD_SIZE")
    if ws_env is None and args.gpus > 1:
        # launched without a launcher: one rank per GPU on this node
        codes = spawn_ranks(args.gpus, [sys.executable, os.path.abspath(__file__),
                                        *(argv if argv is not None else sys.argv[1:])])
        return max(abs(c) for c in codes)
    if ws_env is not None and int(ws_env) != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={ws_env}", file=sys.stderr)
        return 2
    if args.impl == "reference":
        return reference_arm(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
