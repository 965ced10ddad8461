"""Compact state rows (ibgpu_set_state_rows(IBGPU_ROWS_COMPACT)): (roe, u,
v, p) per cell in and out.  An upload derives T and e as the reference
derives them from those four (Get_T_ideal_gas T = p / (roe Rg), Get_E
e = Cv T + |u|^2 / 2, FlowVariables.H:19-33), bit for bit; a download
returns the four fields of the full rows; a step from compact rows equals
the step from the full rows those four imply; the asynchronous pipeline
moves compact rows too."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def implied_rows(P, rows4):
    """The full FlowVariables rows the reference would derive from (roe, u, v, p)."""
    roe, u, v, p = (rows4[:, k].copy() for k in range(4))
    T = p / (roe * P["Rg"])
    e = P["Cv"] * T + 0.5 * ((u * u + v * v) + 0.0 * 0.0)
    return np.stack([roe, u, v, np.zeros_like(u), p, T, e], axis=1)


def test_compact_rows_round_trip_and_step(cuda_lib, pkg):
    ib, wl = pkg.ibgpu, pkg.workloads
    n = 64
    P, cells, prim = wl.vortex_case(n, precision=ib.FP64_EXACT)
    rows4 = np.ascontiguousarray(prim[:, [0, 1, 2, 4]])
    full = implied_rows(P, rows4)

    a = ib.FlowSolver(P)
    a.upload_topology(**cells)
    a.set_state_rows(ib.ROWS_COMPACT)
    a.init_flow(rows4)
    a.set_state_rows(ib.ROWS_FLOWVARS)
    assert np.array_equal(a.download(), full)  # T and e derived bit for bit
    b = ib.FlowSolver(P)
    b.upload_topology(**cells)
    b.init_flow(full)
    for ts in range(2):
        a.time_marching(ts)
        b.time_marching(ts)
    a.set_state_rows(ib.ROWS_COMPACT)
    got4 = a.download()
    want = b.download()
    assert got4.shape == (n * n, 4)
    assert np.array_equal(got4, want[:, [0, 1, 2, 4]])
    a.close()
    b.close()


def test_compact_rows_through_the_asynchronous_pipeline(cuda_lib, pkg):
    import torch
    ib, wl = pkg.ibgpu, pkg.workloads
    n = 64
    P, cells, prim = wl.vortex_case(n, precision=ib.FP64)
    rows4 = np.ascontiguousarray(prim[:, [0, 1, 2, 4]])
    ref = ib.FlowSolver(P)
    ref.upload_topology(**cells)
    ref.init_flow(implied_rows(P, rows4))
    outs = []
    for s in range(3):
        ref.time_marching(s)
        outs.append(ref.download()[:, [0, 1, 2, 4]])
        ref.init_flow(implied_rows(P, rows4))  # every step restarts from the same rows
    ref.close()
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.set_state_rows(ib.ROWS_COMPACT)
    sol.init_flow(rows4)
    host_in = torch.from_numpy(rows4).pin_memory()
    host_out = [torch.empty_like(host_in).pin_memory() for _ in range(3)]
    for s in range(3):
        sol.upload_async(host_in.data_ptr())
        sol.step_async(s)
        sol.download_async(host_out[s].data_ptr())
    sol.step_result()
    sol.synchronize()
    for s in range(3):
        assert np.array_equal(host_out[s].numpy(), outs[s]), s
    sol.close()
