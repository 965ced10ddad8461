"""Run a few time steps of a workload through the C ABI, for profilers.

    python immsered-boundary_b200/profile_step.py --n 2048 --steps 4 --precision fp64

Builds the periodic isentropic-vortex case of the given size and runs
``--steps`` full time steps (4 stages each) on cuda:0; prints the mean step
time.  Used as the command under ``ncu`` (the kernel of interest is
``stage_kernel``).
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))


def _pkg():
    name = "immsered_boundary_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "exact", "mixed"])
    ap.add_argument("--limiter", default="vanleer", choices=["vanleer", "minmod"])
    ap.add_argument("--batch", type=int, default=0,
                    help="instead: this many batched vortex cases (50k..800k cells, seed 0)")
    ap.add_argument("--grid", type=int, default=-1,
                    help="batched: CTA count of the merged launches (0 one per item, "
                         "-1 autotuned)")
    a = ap.parse_args()
    pkg = _pkg()
    ib, wl = pkg.ibgpu, pkg.workloads
    prec = {"fp64": ib.FP64, "exact": ib.FP64_EXACT, "mixed": ib.MIXED}[a.precision]
    if a.batch:
        sols = []
        for P, cells, prim in wl.batch_vortex_cases(a.batch, seed=0, precision=prec):
            s = ib.FlowSolver(P)
            s.upload_topology(**cells)
            s.init_flow(prim)
            sols.append(s)
        b = ib.Batch(sols)
        b.set_grid(a.grid)
        b.run(0, 1)
        t0 = time.perf_counter()
        b.run(1, a.steps)
        dt = (time.perf_counter() - t0) / max(a.steps, 1)
        ncell = sum(s.ncells for s in sols)
        print(f"batch of {a.batch} cases ({ncell} cells) {a.precision}: {dt * 1e3:.3f} ms/step "
              f"({ncell / dt / 1e9:.2f} G cell-updates/s, wall), {b.info()}")
        b.close()
        for s in sols:
            s.close()
        return
    lim = ib.LIM_VANLEER if a.limiter == "vanleer" else ib.LIM_MINMOD
    P, cells, prim = wl.vortex_case(a.n, limiter=lim, precision=prec)
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.init_flow(prim)
    sol.time_marching(0)
    t0 = time.perf_counter()
    sol.run(1, a.steps)
    dt = (time.perf_counter() - t0) / max(a.steps, 1)
    print(f"{a.n}x{a.n} {a.precision}: {dt * 1e3:.3f} ms/step (wall, {a.steps} steps back to back)")
    sol.close()


if __name__ == "__main__":
    main()
