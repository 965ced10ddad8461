"""Batched cases (ibgpu_batch_*): several independent cases advanced by one
merged, graph-replayed launch per stage give bit for bit the same states as
the same cases stepped one by one."""
import os
import sys

import numpy as np
import pytest

from conftest import load_pkg

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402

pytestmark = pytest.mark.gpu

pkg = load_pkg()
ib, wl = pkg.ibgpu, pkg.workloads


def make_solver(case):
    P, cells, prim = case
    s = ib.FlowSolver(P)
    s.upload_topology(**cells)
    s.init_flow(prim)
    return s


@pytest.mark.parametrize("precision", [ib.FP64, ib.MIXED])
def test_batched_vortex_cases_equal_single_runs(cuda_lib, precision):
    cases = [wl.vortex_case(n, precision=precision, mach=m, angle_deg=a)
             for n, m, a in [(64, 0.5, 45.0), (96, 0.2, 0.0), (48, 0.8, -5.0)]]
    single = [make_solver(c) for c in cases]
    for s in single:
        s.run(0, 5)
    batched = [make_solver(c) for c in cases]
    b = ib.Batch(batched)
    b.run(0, 2)
    d = b.run(2, 3)
    for s, t, di in zip(single, batched, d):
        assert t.dt == s.dt
        assert np.array_equal(t.download(), s.download())
        assert di.abort_code == 0 and di.cells_marched > 0
    info = b.info()
    assert info["period"] == 1 and len(info["tuning"]) >= 1
    assert info["table_bytes"] > 0  # arguments read from the constant-memory table
    b.close()
    for s in single + batched:
        s.close()


@pytest.mark.parametrize("grid", [0, 3])
def test_batch_fixed_cta_counts_equal_single_runs(cuda_lib, grid):
    """One CTA per work item and a persistent grid of 3 CTAs (each strides
    over many items) set by the caller instead of the autotuner."""
    cases = [wl.vortex_case(n, precision=ib.MIXED, mach=m) for n, m in [(64, 0.4), (32, 0.7)]]
    single = [make_solver(c) for c in cases]
    for s in single:
        s.run(0, 3)
    batched = [make_solver(c) for c in cases]
    b = ib.Batch(batched)
    b.set_grid(grid)
    b.run(0, 3)
    info = b.info()
    # the block shape is still tuned, at the caller's CTA count
    assert info["grid"] == grid and {t[0] for t in info["tuning"]} == {grid}
    assert {t[1] for t in info["tuning"]} == {256, 288}
    for s, t in zip(single, batched):
        assert t.dt == s.dt
        assert np.array_equal(t.download(), s.download())
    with pytest.raises(ib.IbgpuError):
        b.set_grid(-2)
    b.close()
    for s in single + batched:
        s.close()


@pytest.mark.parametrize("precision", [ib.FP64, ib.MIXED])
@pytest.mark.parametrize("threads", [256, 288])
def test_batch_block_shapes_equal_single_runs(cuda_lib, precision, threads):
    """Both block shapes of the merged stage launch (the tile's edge faces
    on the first two warps, or on a ninth warp), fixed by the caller, with
    one CTA per item and with persistent CTAs: the cases' bits alone."""
    cases = [wl.vortex_case(n, precision=precision, mach=m) for n, m in [(64, 0.4), (48, 0.7)]]
    single = [make_solver(c) for c in cases]
    for s in single:
        s.run(0, 4)
    for grid in (0, 5):
        batched = [make_solver(c) for c in cases]
        b = ib.Batch(batched)
        b.set_block(threads)
        b.set_grid(grid)
        b.run(0, 4)
        info = b.info()
        assert info["threads"] == threads and info["grid"] == grid and info["tuning"] == []
        for s, t in zip(single, batched):
            assert t.dt == s.dt
            assert np.array_equal(t.download(), s.download())
        with pytest.raises(ib.IbgpuError):
            b.set_block(128)
        b.close()
        for t in batched:
            t.close()
    for s in single:
        s.close()


@pytest.mark.parametrize("precision", [ib.FP64, ib.MIXED])
def test_batch_beyond_constant_table_reads_global_arguments(cuda_lib, precision):
    """88 small cases need more than the 60 KiB constant-memory argument
    table: the batch falls back to arguments in global memory and still
    equals the cases stepped alone; a small batch created beside it gets
    table space and agrees too."""
    cases = [wl.vortex_case(16 * (1 + i % 3), precision=precision, mach=0.2 + 0.007 * i,
                            angle_deg=float(i % 11)) for i in range(90)]
    ref = []
    for c in cases:
        s = make_solver(c)
        s.run(0, 3)
        ref.append((s.dt, s.download()))
        s.close()
    sols = [make_solver(c) for c in cases]
    big = ib.Batch(sols[:88])  # about 752 bytes of table per case
    small = ib.Batch(sols[88:])
    assert big.info()["table_bytes"] == 0
    assert small.info()["table_bytes"] > 0
    big.run(0, 3)
    small.run(0, 3)
    for s, (dt, prim) in zip(sols, ref):
        assert s.dt == dt
        assert np.array_equal(s.download(), prim)
    big.close()
    small.close()
    for s in sols:
        s.close()


def test_batched_amr_cases_follow_their_own_schedules(cuda_lib):
    """Two 3-level NACA cases (immersed body, viscous, subcycling) started
    from different reference states, batched for a full subcycling period,
    against the same cases stepped alone: the merged work lists follow each
    case's marching levels step by step."""
    g = make_golden.load("naca_minmod_s4_n64_l3")
    with pytest.raises(ib.IbgpuError):
        ib.Batch([])
    # case A starts from the initial state and first catches up to step 2
    a = wl.naca_solver(g, 0, ib.FP64)
    a.run(0, 2)
    bcase = wl.naca_solver(g, 2, ib.FP64)
    batch = ib.Batch([a, bcase])
    assert batch.info()["period"] == 4
    batch.run(2, 4)
    ra = wl.naca_solver(g, 0, ib.FP64)
    ra.run(0, 2)
    ra.run(2, 4)
    rb = wl.naca_solver(g, 2, ib.FP64)
    rb.run(2, 4)
    for t, s in ((a, ra), (bcase, rb)):
        assert t.dt == s.dt
        assert np.array_equal(t.download(), s.download())
        assert np.array_equal(t.wall_forces(), s.wall_forces())
    batch.close()
    for s in (a, bcase, ra, rb):
        s.close()


def test_batch_tag_mesh_equals_per_case_tagging(cuda_lib):
    import torch
    cases = [wl.vortex_case(n, mach=m) for n, m in [(64, 0.5), (48, 0.3)]]
    sols = [make_solver(c) for c in cases]
    rule = wl.naca_tag_rule(1, [10.0 / 64])
    params = torch.from_numpy(pkg.indicator.init_params(3)).cuda()
    b = ib.Batch(sols)
    for dp in (0, params.data_ptr()):
        got = b.tag_mesh(rule, dp)
        for s, g in zip(sols, got):
            assert np.array_equal(g, s.tag_mesh(rule, dp))
    b.close()
    for s in sols:
        s.close()


def test_batched_cases_with_different_cfl_intervals(cuda_lib):
    """A 3-level and a 4-level airfoil case (CFL pass every 4 and every 8
    steps: the reference rounds dt_var_step up to the coarsest level's step)
    in one batch for two schedule periods, against each case stepped alone:
    each case takes its CFL pass on its own steps."""
    g3 = make_golden.load("naca_minmod_s4_n64_l3")
    g4 = make_golden.load("naca_minmod_s4_n128_l4")
    dvs = [int(g["scalars"][0][15 + int(g["scalars"][0][14])]) for g in (g3, g4)]
    assert dvs[0] != dvs[1]
    sols = [wl.naca_solver(g, 0, ib.FP64) for g in (g3, g4)]
    batch = ib.Batch(sols)
    assert batch.info()["period"] == 8
    batch.run(0, 16)
    for s, g in zip(sols, (g3, g4)):
        r = wl.naca_solver(g, 0, ib.FP64)
        r.run(0, 16)
        assert s.dt == r.dt
        assert np.array_equal(s.download(), r.download())
        r.close()
    batch.close()
    for s in sols:
        s.close()
