"""Train the learned refinement indicator for a few steps on synthetic rows,
for profilers (the kernel of interest is ``mlp_grad_kernel``).

    python immsered-boundary_b200/profile_indicator.py --rows 262144 --steps 5

Rows are random BF16 features with random labels (the kernel's work does not
depend on the values); prints the mean time of one training step.
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import sys
import time

import numpy as np

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
    ap.add_argument("--rows", type=int, default=262144)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--mesh", type=int, default=0,
                    help="instead: learned tagging of every cell of an N x N vortex case")
    a = ap.parse_args()
    if a.mesh:
        return mesh_tagging(a.mesh, a.steps)
    import torch
    pkg = _pkg()
    ib, ind, wl = pkg.ibgpu, pkg.indicator, pkg.workloads
    P, cells, prim = wl.vortex_case(64)
    sol = ib.FlowSolver(P)
    rng = np.random.default_rng(0)
    X = rng.normal(0, 1, (a.rows, ib.MLP_IN)).astype(np.float32)
    bits = (X.view(np.uint32) >> 16).astype(np.uint16)
    feat = torch.from_numpy(bits.view(np.int16)).cuda()
    y = rng.integers(0, 3, a.rows).astype(np.uint8)
    li = ind.LearnedIndicator(sol, seed=0)
    li.train(feat, y, steps=2, batch=a.rows)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    li.train(feat, y, steps=a.steps, batch=a.rows)
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / a.steps
    print(f"{a.rows} rows: {dt * 1e3:.3f} ms per training step (wall, incl. host sync)")
    sol.close()


def mesh_tagging(n: int, reps: int):
    """ibgpu_tag_mesh (learned) on every cell of an n x n case; the kernel
    of interest is ``mlp_tag_mesh_kernel``."""
    import torch
    pkg = _pkg()
    ib, ind, wl = pkg.ibgpu, pkg.indicator, pkg.workloads
    P, cells, prim = wl.vortex_case(n)
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.init_flow(prim)
    li = ind.LearnedIndicator(sol, seed=0)
    rule = wl.naca_tag_rule(1, [10.0 / n])
    sol.tag_mesh(rule, li.params.data_ptr())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        tags = sol.tag_mesh(rule, li.params.data_ptr())
    dt = (time.perf_counter() - t0) / reps
    print(f"{n}x{n}: {dt * 1e3:.3f} ms per ibgpu_tag_mesh call ({n * n / dt / 1e9:.3f} G cells/s), "
          f"tag counts {np.bincount(tags, minlength=4).tolist()}")
    sol.close()


if __name__ == "__main__":
    main()
