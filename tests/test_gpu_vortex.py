"""GPU step parity on the periodic isentropic-vortex workload.

* against the reference solver's own dumps (golden fixtures): the exact-FP64
  build must reproduce every step bit for bit, the FP64 build within 1e-12
  relative on the conserved variables per step, the mixed build within its
  stated FP32-flux tolerance;
* against the CPU oracle on larger grids and several consecutive steps;
* size-independent properties at the full 2048 x 2048 size (discrete
  conservation of mass, momentum and energy on the periodic grid);
* the reference's abort conditions and the ABI's argument/topology errors.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402

pytestmark = pytest.mark.gpu

GOLDEN = [("vortex_vanleer_s4_n32", 0), ("vortex_minmod_s3_n32", 1)]
REL_FP64 = 1e-12   # conserved variables, relative to the field's max magnitude, per step
REL_MIXED = 2e-5   # FP32 flux / limiter, FP64 accumulation, per step


def params_from_golden(ib, g, k, limiter, precision, viscous=False):
    s = g["scalars"][k]
    nst = int(s[14])
    dom = g["domain"]
    nlev = int(dom[5])
    sched = g["schedule"].reshape(-1, 6)
    dh = g["dh"].reshape(-1, 3)
    return dict(gama=s[4], Rg=s[5], Cv=s[6], Cp=s[7], Ma=s[8], Re=s[9], Pr=s[10], qk=s[11],
                s_over_t=s[12], cfl=s[13], nstages=nst, tp=list(s[15:15 + nst]),
                dt_ratio=1.0, dt_var_step=1, limiter=limiter, viscous=int(viscous),
                precision=precision, initvar=list(g["initvar"]), nlevels=nlev,
                dh=[tuple(dh[l]) for l in range(nlev)],
                march_step=[int(sched[l, 0]) for l in range(nlev)],
                march_left=[int(sched[l, 3]) for l in range(nlev)],
                step_num=[float(sched[l, 0]) for l in range(nlev)],
                domain_nx=int(dom[0]), domain_ny=int(dom[1]), periodic_x=int(dom[2]),
                periodic_y=int(dom[3]), dt0=float(s[1]))


def solver_from_golden(ib, g, k, limiter, precision):
    P = params_from_golden(ib, g, k, limiter, precision)
    sol = ib.FlowSolver(P)
    body_level = int(g["domain"][4]) > 0
    flags = np.zeros(len(g["level"]), np.uint8)
    for l in range(P["nlevels"]):
        m = g["level"] == l
        flags[m] = ib.cell_flags_from_boxes(g["kind"][m], g["solid"][m], g["infect"][m],
                                            g["signdis"][m], body_level and l == P["nlevels"] - 1)
    sol.upload_topology(g["level"], g["ix"], g["iy"], flags)
    sol.init_flow(g["prim"][k])
    return sol, flags


def conserved(prim):
    r, u, v, e = prim[:, 0], prim[:, 1], prim[:, 2], prim[:, 6]
    return np.stack([r, r * u, r * v, r * e], axis=1)


def rel_err(got, ref):
    cg, cr = conserved(got), conserved(ref)
    scale = np.abs(cr).max(axis=0)
    return (np.abs(cg - cr).max(axis=0) / scale).max()


@pytest.mark.parametrize("name,limiter", GOLDEN)
def test_exact_build_reproduces_reference_bitwise(cuda_lib, pkg, name, limiter):
    ib = pkg.ibgpu
    g = make_golden.load(name)
    keep = g["kind"] != ib.BOX_BLOCK_GHOST  # block ghosts are refreshed at the next exchange
    for k in range(g["prim"].shape[0] - 1):
        sol, _ = solver_from_golden(ib, g, k, limiter, ib.FP64_EXACT)
        d = sol.time_marching(k)
        assert d.abort_code == 0
        assert sol.dt == g["scalars"][k + 1][1]
        got = sol.download()
        ref = g["prim"][k + 1]
        bad = np.flatnonzero(np.any(got[keep] != ref[keep], axis=1))
        assert bad.size == 0, f"step {k}: {bad.size} cells differ, max {np.abs(got - ref)[keep].max()}"
        sol.close()


@pytest.mark.parametrize("name,limiter", GOLDEN)
def test_fp64_build_within_1e12(cuda_lib, pkg, name, limiter):
    ib = pkg.ibgpu
    g = make_golden.load(name)
    keep = g["kind"] == ib.BOX_NORMAL
    for k in range(g["prim"].shape[0] - 1):
        sol, _ = solver_from_golden(ib, g, k, limiter, ib.FP64)
        sol.time_marching(k)
        got = sol.download()
        assert rel_err(got[keep], g["prim"][k + 1][keep]) <= REL_FP64
        sol.close()


@pytest.mark.parametrize("name,limiter", GOLDEN)
def test_mixed_build_within_stated_tolerance(cuda_lib, pkg, name, limiter):
    ib = pkg.ibgpu
    g = make_golden.load(name)
    keep = g["kind"] == ib.BOX_NORMAL
    errs = []
    for k in range(g["prim"].shape[0] - 1):
        sol, _ = solver_from_golden(ib, g, k, limiter, ib.MIXED)
        sol.time_marching(k)
        got = sol.download()
        errs.append(rel_err(got[keep], g["prim"][k + 1][keep]))
        sol.close()
    assert max(errs) <= REL_MIXED, errs


def oracle_levels_for(oracle, ix, iy, prim, n, params):
    """Dense oracle arrays for a single periodic level of n x n leaf cells
    plus the reference's two block-ghost layers."""
    ghosts_x, ghosts_y = [], []
    for y in range(-2, n + 2):
        for x in range(-2, n + 2):
            if x < 0 or y < 0 or x >= n or y >= n:
                ghosts_x.append(x)
                ghosts_y.append(y)
    gx = np.array(ghosts_x, np.int32)
    gy = np.array(ghosts_y, np.int32)
    d = dict(level=np.concatenate([np.zeros_like(ix), np.zeros_like(gx)]),
             ix=np.concatenate([ix, gx]), iy=np.concatenate([iy, gy]),
             kind=np.concatenate([np.zeros_like(ix), np.full_like(gx, 2)]),
             ptype=np.zeros(len(ix) + len(gx), np.int32), solid=np.zeros(len(ix) + len(gx), np.int32),
             infect=np.full(len(ix) + len(gx), -1, np.int32),
             signdis=np.full(len(ix) + len(gx), 9999.0),
             prim=np.concatenate([prim, prim[(gy % n) * n + (gx % n)]]).ravel(),
             dh=np.array(params["dh"][0], np.float64),
             schedule=np.array([1, 2, 2, 0, 1, 1], np.int32),
             domain=np.array([n, n, 1, 1, 0, 1], np.int32),
             initvar=np.array(params["initvar"]))
    return d, oracle.OracleLevels(d)


@pytest.mark.parametrize("limiter", [0, 1])
def test_multistep_against_oracle_64(cuda_lib, pkg, oracle, limiter):
    ib, wl = pkg.ibgpu, pkg.workloads
    n = 64
    P, cells, prim = wl.vortex_case(n, nstages=4, limiter=limiter, precision=ib.FP64_EXACT)
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.init_flow(prim)
    d, lv = oracle_levels_for(oracle, cells["ix"], cells["iy"], prim, n, P)
    OP = dict(P)
    OP["limiter"] = limiter
    dt_o = 1.0
    for ts in range(6):
        diag = sol.time_marching(ts)
        rc, dt_o, cfl, res = oracle.step(OP, lv, ts, dt_o)
        assert rc == 0 and diag.abort_code == 0
        assert sol.dt == dt_o
        assert list(diag.res_max) == res
    got = sol.download()
    ref = lv.state_like_dump(d)[: n * n]
    assert np.array_equal(got, ref)


def test_full_size_conservation_2048(cuda_lib, pkg):
    """Periodic finite-volume update: total mass, momentum and energy change
    only by rounding (size-independent property at the benchmark size)."""
    ib, wl = pkg.ibgpu, pkg.workloads
    n = 2048
    P, cells, prim = wl.vortex_case(n, nstages=4, precision=ib.FP64)
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.init_flow(prim)
    c0 = conserved(prim).sum(axis=0)
    for ts in range(3):
        d = sol.time_marching(ts)
        assert d.abort_code == 0 and d.cells_marched == n * n
    got = sol.download()
    assert np.isfinite(got).all()
    c1 = conserved(got).sum(axis=0)
    scale = np.abs(conserved(prim)).sum(axis=0)
    assert (np.abs(c1 - c0) / scale).max() < 1e-12
    sol.close()


def test_full_size_one_step_matches_oracle_2048(cuda_lib, pkg, oracle):
    ib, wl = pkg.ibgpu, pkg.workloads
    n = 2048
    P, cells, prim = wl.vortex_case(n, nstages=4, precision=ib.FP64_EXACT)
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.init_flow(prim)
    sol.time_marching(0)
    got = sol.download()
    d, lv = oracle_levels_for(oracle, cells["ix"], cells["iy"], prim, n, P)
    rc, dt_o, _, _ = oracle.step(P, lv, 0, 1.0)
    assert rc == 0 and dt_o == sol.dt
    ref = lv.state_like_dump(d)[: n * n]
    assert np.array_equal(got, ref)
    sol.close()


def test_mixed_vs_fp64_full_size_error_is_small(cuda_lib, pkg):
    ib, wl = pkg.ibgpu, pkg.workloads
    n = 512
    out = {}
    for prec in (ib.FP64, ib.MIXED):
        P, cells, prim = wl.vortex_case(n, precision=prec)
        sol = ib.FlowSolver(P)
        sol.upload_topology(**cells)
        sol.init_flow(prim)
        for ts in range(20):
            sol.time_marching(ts)
        out[prec] = sol.download()
        sol.close()
    l2 = np.sqrt(np.mean((out[ib.MIXED][:, 0] - out[ib.FP64][:, 0]) ** 2))
    assert l2 < 1e-5, l2


@pytest.mark.parametrize("dt,expect", [(1.0, 523), (10.0, 37)])
def test_abort_codes_match_the_reference_order(cuda_lib, pkg, oracle, dt, expect):
    """An over-large dt (no CFL evaluation on this step) drives the update
    invalid; the GPU reports the same abort as the reference's sequential
    order: every density check of a stage (523) before any temperature check
    (37)."""
    ib, wl = pkg.ibgpu, pkg.workloads
    n = 32
    P, cells, prim = wl.vortex_case(n, precision=ib.FP64_EXACT)
    P["dt_var_step"] = 2
    P["dt0"] = dt
    d, lv = oracle_levels_for(oracle, cells["ix"], cells["iy"], prim, n, P)
    rc, *_ = oracle.step(P, lv, 1, dt)
    assert rc == expect
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.init_flow(prim)
    with pytest.raises(ib.IbgpuError) as ei:
        sol.time_marching(1)
    assert ei.value.code == ib.E_ABORT
    assert ei.value.abort_code == expect
    assert ei.value.diag.abort_level == 0
    sol.close()


def test_blown_out_cell_aborts_on_temperature(cuda_lib, pkg, oracle):
    ib, wl = pkg.ibgpu, pkg.workloads
    n = 32
    P, cells, prim = wl.vortex_case(n, precision=ib.FP64_EXACT)
    bad = prim.copy()
    c = 10 * n + 10
    bad[c, 0] = 1e-9                       # an almost empty cell ...
    bad[c, 1] = 50.0                       # ... blown out by a strong outflow
    bad[c, 6] = P["Cv"] * bad[c, 5] + 0.5 * bad[c, 1] ** 2
    d, lv = oracle_levels_for(oracle, cells["ix"], cells["iy"], bad, n, P)
    rc, *_ = oracle.step(P, lv, 0, 1.0)
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.init_flow(bad)
    with pytest.raises(ib.IbgpuError) as ei:
        sol.time_marching(0)
    assert ei.value.abort_code == rc == 37
    sol.close()


def test_nan_state_reports_nan_residual(cuda_lib, pkg, oracle):
    """A NaN in the state propagates identically, and the GPU reports it as
    the NaN-residual abort (268).  Deliberately stricter than the reference:
    its max-norm fold std::max(|s|, acc) (NS_Solver.H:302-307) drops a NaN
    unless it sits in the last cell of the loop, so the reference (and the
    oracle that restates it) usually carries on with the NaN state."""
    ib, wl = pkg.ibgpu, pkg.workloads
    n = 32
    P, cells, prim = wl.vortex_case(n, precision=ib.FP64_EXACT)
    bad = prim.copy()
    bad[5 * n + 7, 4] = np.nan
    d, lv = oracle_levels_for(oracle, cells["ix"], cells["iy"], bad, n, P)
    rc, *_ = oracle.step(P, lv, 0, 1.0)
    ref = lv.state_like_dump(d)[: n * n]
    assert rc == 0 and np.isnan(ref).any()
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.init_flow(bad)
    with pytest.raises(ib.IbgpuError) as ei:
        sol.time_marching(0)
    assert ei.value.abort_code == 268
    got = sol.download()
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    ok = ~np.isnan(ref)
    assert np.array_equal(got[ok], ref[ok])
    sol.close()


def test_topology_errors(cuda_lib, pkg):
    ib, wl = pkg.ibgpu, pkg.workloads
    # periodic extent that is not a multiple of the 16-cell tile
    P, cells, prim = wl.vortex_case(40)
    sol = ib.FlowSolver(P)
    with pytest.raises(ib.IbgpuError) as ei:
        sol.upload_topology(**cells)
    assert ei.value.code == ib.E_TOPOLOGY
    # two cells at one position
    P, cells, prim = wl.vortex_case(32)
    sol = ib.FlowSolver(P)
    dup = {k: np.concatenate([v, v[:1]]) for k, v in cells.items()}
    with pytest.raises(ib.IbgpuError) as ei:
        sol.upload_topology(**dup)
    assert ei.value.code == ib.E_TOPOLOGY
    # a leaf cell without its face neighbour (non-periodic level, no ghosts)
    P2 = dict(P, periodic_x=0, periodic_y=0)
    sol = ib.FlowSolver(P2)
    with pytest.raises(ib.IbgpuError) as ei:
        sol.upload_topology(**cells)
    assert ei.value.code == ib.E_TOPOLOGY
    assert "missing face neighbour" in str(ei.value)
    # a west face whose outer MUSCL neighbours are both missing: a column of
    # leaves with one ghost column to the west and nothing to the east
    leaf = ib.CELL_PRESENT | ib.CELL_NORMAL | ib.CELL_UPDATE | ib.CELL_PRIM | ib.CELL_RESNORM
    lv, xs, ys, fl = [], [], [], []
    for iy in range(32):
        for ix, f in ((-1, ib.CELL_PRESENT), (0, leaf)):
            lv.append(0)
            xs.append(ix)
            ys.append(iy)
            fl.append(f)
    sol = ib.FlowSolver(P2)
    with pytest.raises(ib.IbgpuError) as ei:
        sol.upload_topology(np.array(lv), np.array(xs), np.array(ys), np.array(fl))
    assert ei.value.code == ib.E_TOPOLOGY
    assert "neither outer neighbour" in str(ei.value)
    # step before any state
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    with pytest.raises(ib.IbgpuError) as ei:
        sol.time_marching(0)
    assert ei.value.code == ib.E_STATE
    # an empty mesh steps as a no-op
    sol = ib.FlowSolver(P)
    sol.upload_topology(level=[], ix=[], iy=[], flags=[])
    sol.init_flow(np.zeros((0, 7)))
    d = sol.time_marching(0)
    assert d.cells_marched == 0


def test_run_equals_single_steps_and_reports_abort_step(cuda_lib, pkg):
    """ibgpu_run (steps back to back, dt kept on the device) gives exactly the
    state of the same number of single ibgpu_step calls, and reports an
    abort with the index of the step that hit it."""
    ib, wl = pkg.ibgpu, pkg.workloads
    n = 64
    P, cells, prim = wl.vortex_case(n, precision=ib.FP64)
    a = ib.FlowSolver(P)
    a.upload_topology(**cells)
    a.init_flow(prim)
    for ts in range(5):
        a.time_marching(ts)
    b = ib.FlowSolver(P)
    b.upload_topology(**cells)
    b.init_flow(prim)
    d = b.run(0, 5)
    assert d.abort_code == 0 and b.dt == a.dt
    assert np.array_equal(a.download(), b.download())
    # over-large dt from step 1 on (CFL evaluated only every 4 steps): the
    # first step is fine, a later one aborts
    P2 = dict(P, dt_var_step=4)
    c = ib.FlowSolver(P2)
    c.upload_topology(**cells)
    c.init_flow(prim)
    c.dt = 1.0
    with pytest.raises(ib.IbgpuError) as ei:
        c.run(1, 3)
    assert ei.value.abort_code in (523, 37)
    assert ei.value.diag.abort_step == 0


def test_async_download_is_ordered_with_later_uploads(cuda_lib, pkg):
    """ibgpu_download_state_async returns before the copy ends; an upload and
    a step issued right after must not disturb the state it copies."""
    import torch
    ib, wl = pkg.ibgpu, pkg.workloads
    P, cells, prim = wl.vortex_case(64)
    ref = ib.FlowSolver(P)
    ref.upload_topology(**cells)
    ref.init_flow(prim)
    ref.time_marching(0)
    want = ref.download()
    ref.close()
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.init_flow(prim)
    sol.time_marching(0)
    out = torch.empty((len(prim), 7), dtype=torch.float64).pin_memory()
    sol.download_async(out.data_ptr())
    other = prim.copy()
    other[:, 4] *= 1.01  # a different state uploaded while the copy may run
    sol.init_flow(other)
    sol.time_marching(1)
    sol.synchronize()
    assert np.array_equal(out.numpy(), want)
    sol.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pipelined_steps_equal_synchronous_steps(cuda_lib, pkg, precision):
    """ibgpu_upload_state_async + ibgpu_step_async + ibgpu_download_state_async
    for several steps, each from its own uploaded state, with one host wait at
    the end: every step's result and the final dt and diag equal the
    synchronous calls' bit for bit."""
    import torch
    ib, wl = pkg.ibgpu, pkg.workloads
    prec = {"fp64": ib.FP64, "mixed": ib.MIXED}[precision]
    P, cells, prim = wl.vortex_case(64, precision=prec)
    K = 4
    inputs = []
    for k in range(K):
        q = prim.copy()
        q[:, 4] *= 1.0 + 0.01 * k  # every step starts from its own state
        inputs.append(q)
    ref = ib.FlowSolver(P)
    ref.upload_topology(**cells)
    want, dts = [], []
    for k in range(K):
        ref.init_flow(inputs[k])
        d_ref = ref.time_marching(k)
        dts.append(ref.dt)
        want.append(ref.download())
    ref.close()
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    host_in = [torch.from_numpy(q).pin_memory() for q in inputs]
    host_out = [torch.empty_like(h).pin_memory() for h in host_in]
    for k in range(K):
        sol.upload_async(host_in[k].data_ptr())
        sol.step_async(k)
        sol.download_async(host_out[k].data_ptr())
    d = sol.step_result()
    sol.synchronize()
    for k in range(K):
        assert np.array_equal(host_out[k].numpy(), want[k]), k
    assert sol.dt == dts[-1]
    assert d.abort_code == 0 and d.cells_marched == d_ref.cells_marched
    assert list(d.res_max) == list(d_ref.res_max)
    # no result without a chain; no synchronous step while one is open
    with pytest.raises(ib.IbgpuError):
        sol.step_result()
    sol.step_async(K)
    with pytest.raises(ib.IbgpuError):
        sol.time_marching(K + 1)
    sol.step_result()
    sol.close()
