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
REF_SAMPLE_N = 1024  # bounded CPU sample: 1024 x 1024 cells of the same case


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


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name="stage_kernel_vortex2048.txt"):
    """dram bytes per stage launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, flags in rows for i, f in enumerate(flags)
                          if f.lower() == "active"})
        mx = max(r[1] for r in rows)
        loaded = [r[0] for r in rows if r[0] > 0.5 * mx] or [r[0] for r in rows]
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def reference_binary():
    p = os.path.join(ROOT, "oracle", "_ref", "ref_vortex_vanleer")
    return p if os.path.exists(p) and os.access(p, os.X_OK) else None


def run_reference(n: int, steps: int, warmup: int = 0):
    """The reference solver's own step (compiled from its sources with the
    single-rank MPI shim) on the host: returns (cell_updates_per_s, seconds,
    cell_updates, kind).  Falls back to the C restatement (kind "port") when
    the reference build is absent."""
    binary = reference_binary()
    if binary is not None:
        env = dict(os.environ, IB_NX=str(n), IB_STEPS=str(steps), IB_STAGES=str(STAGES),
                   IB_TIMED_FROM=str(warmup))
        with tempfile.TemporaryDirectory() as wd:
            out = subprocess.run([binary], cwd=wd, env=env, capture_output=True, text=True,
                                 check=True).stdout
        for line in out.splitlines():
            if line.startswith("ORACLE_RESULT"):
                r = json.loads(line.split(" ", 1)[1])
                return r["cell_updates_per_s"], r["loop_seconds"], r["cell_updates"], "reference"
        raise RuntimeError("reference run printed no result")
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
    return upd / sec, sec, upd, "port"


def reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    n = REF_SAMPLE_N
    rate, sec, upd, kind = run_reference(n, args.warmup + args.steps, args.warmup)
    sample = (f"{args.steps} timed steps (after {args.warmup} warm-up) of the same case on a "
              f"{n}x{n} grid ({n * n} leaf cells per step), step loop only")
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3 / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"isentropic vortex {N_DEFAULT}x{N_DEFAULT} periodic, inviscid, "
                               "4-stage, VanLeer MUSCL, all-speed Roe, CFL 0.5",
                   "sample_grid": f"{n}x{n}", "parallelism": "replicas"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 1, "kind": kind, "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


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
    ms, clocks = timed_steps(sol, args.warmup, args.steps, sampler)
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
    # the state, steps, and reads the state back
    host_in = torch.from_numpy(prim.astype(np.float64)).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    e2e_steps = max(3, min(args.steps, 10))
    barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    t0 = time.perf_counter()
    for s in range(e2e_steps):
        sol.init_flow(host_in.data_ptr())
        sol.time_marching(s)
        sol.download(host_out.data_ptr())
    ev1.record(stream)
    ev1.synchronize()
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

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        rate, sec, upd, kind = run_reference(REF_SAMPLE_N, 2, 0)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": kind,
               "sample": f"2 time steps of the same case on a {REF_SAMPLE_N}x{REF_SAMPLE_N} grid "
                         f"({upd} leaf-cell updates), step loop only, single-rank build"}

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
            "gpu_launches": (2 + STAGES) * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "stage_kernel (flux + residual + update + prim recovery)",
                         "bytes_per_launch": stage_bytes, "ms_per_launch": stage_ms,
                         "peak_source": peak_kind},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": ncell * 7 * 8,
                    "d2h_bytes_per_step": ncell * 7 * 8,
                    "path": "ibgpu_upload_state + ibgpu_step + ibgpu_download_state per step"},
            "mixed": {"value": mixed_value, "unit": UNIT, "ms_per_step": mms / args.steps,
                      "stage_ms_per_launch": mk[0] / max(mkn[0], 1),
                      "dtype": "f32 flux/limiter, f64 accumulation"},
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
