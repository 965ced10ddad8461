"""The allocation-free step entry point (ibgpu_step_periodic_noalloc).

Callers that may not allocate device memory while they run (a coupler whose
device memory belongs to another framework, a time loop that cannot take
cudaMalloc's device-wide synchronisation) hand the library their own device
buffers; everything else lives in the library's fixed device array.  Here the
test plays that caller: torch owns the in/out buffers, the library allocates
nothing, and two consecutive steps must agree with the regular entry point
(ibgpu_step through a context) within each build's parity tolerance, on a
square and a non-square grid, the second step taking the caller's dt (no CFL
evaluation on that step).  The device's free memory and torch's allocator
must not move across a call, and an invalid update must report the same
abort code as the regular entry point.

Kept in a file of its own that sorts last, so a run that stops at the first
failure has already run every other test.
"""
import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# per-build tolerance against the regular entry point (the same kernels on the
# same values: both FP64 builds are expected to agree bit for bit)
TOL = {"exact": 0.0, "fp64": 1e-12, "mixed": 5e-5}


def prec_of(ib, name):
    return {"exact": ib.FP64_EXACT, "fp64": ib.FP64, "mixed": ib.MIXED}[name]


def regular_steps(ib, P, cells, prim, nsteps):
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.init_flow(prim)
    out = []
    for ts in range(nsteps):
        sol.time_marching(ts)
        out.append((sol.download(), sol.dt))
    sol.close()
    return out


def vortex_rows(wl, nx, ny, precision):
    """A periodic nx x ny vortex (16-cell tiles) in row-major cell order."""
    P, cells, prim = wl.vortex_case(max(nx, ny), nstages=4, precision=precision)
    keep = (cells["ix"] < nx) & (cells["iy"] < ny)
    cells = {k: v[keep] for k, v in cells.items()}
    P = dict(P, domain_nx=nx, domain_ny=ny)
    return P, cells, np.ascontiguousarray(prim[keep])


@pytest.mark.parametrize("precision", ["exact", "fp64", "mixed"])
@pytest.mark.parametrize("nx,ny", [(64, 64), (128, 32)])
def test_noalloc_step_matches_regular_entry_point_twice(cuda_lib, pkg, precision, nx, ny):
    import torch

    ib, wl = pkg.ibgpu, pkg.workloads
    P, cells, prim = vortex_rows(wl, nx, ny, prec_of(ib, precision))
    # dt from the CFL condition on even steps only: the second step runs on
    # the dt the caller passes in
    P["dt_var_step"] = 2
    ref = regular_steps(ib, P, cells, prim, 2)

    rows = torch.from_numpy(prim).to("cuda")
    out = torch.empty_like(rows)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    dt = P["dt0"]
    src = rows
    for ts in range(2):
        # no other object may free device memory meanwhile (a collected
        # context of an earlier test would)
        gc.collect()
        gc.disable()
        try:
            free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
            dt_in = dt
            dt, diag = ib.step_periodic_noalloc(P, ts, nx, ny, src.data_ptr(), out.data_ptr(), dt,
                                                stream)
            free1 = torch.cuda.mem_get_info()[0]
        finally:
            gc.enable()
        if ts > 0:  # the first call on a device may load the library's module
            assert free1 == free0, "the call allocated device memory"
            assert torch.cuda.memory_allocated() == alloc0
            assert dt == dt_in  # no CFL evaluation on this step
        assert diag.abort_code == 0 and diag.cells_marched == nx * ny
        got = out.cpu().numpy()
        want, want_dt = ref[ts]
        assert dt == want_dt
        scale = np.abs(want).max(axis=0)
        scale[scale == 0] = 1.0
        err = (np.abs(got - want).max(axis=0) / scale).max()
        assert err <= TOL[precision], f"step {ts}: {err:.3e}"
        src = out  # the second call steps in place, continuing from the first


def test_noalloc_reports_the_regular_abort(cuda_lib, pkg):
    """An over-large dt on a step without CFL evaluation drives the update
    invalid: the same abort code as the regular entry point, at a cell of
    the grid."""
    import torch

    ib, wl = pkg.ibgpu, pkg.workloads
    n = 32
    P, cells, prim = wl.vortex_case(n, precision=ib.FP64)
    P["dt_var_step"] = 2
    P["dt0"] = 1.0
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.init_flow(prim)
    with pytest.raises(ib.IbgpuError) as want:
        sol.time_marching(1)
    sol.close()
    rows = torch.from_numpy(prim).to("cuda")
    out = torch.empty_like(rows)
    with pytest.raises(ib.IbgpuError) as got:
        ib.step_periodic_noalloc(P, 1, n, n, rows.data_ptr(), out.data_ptr(), 1.0)
    assert got.value.code == want.value.code == ib.E_ABORT
    assert got.value.abort_code == want.value.abort_code == 523
    g = got.value.diag
    assert 0 <= g.abort_ix < n and 0 <= g.abort_iy < n


def test_noalloc_rejects_sizes_beyond_its_array(cuda_lib, pkg):
    import torch

    ib, wl = pkg.ibgpu, pkg.workloads
    n = 272  # 272 * 272 > IBGPU_NOALLOC_MAX_CELLS
    P, cells, prim = wl.vortex_case(n)
    buf = torch.zeros((16, 7), dtype=torch.float64, device="cuda")
    with pytest.raises(ib.IbgpuError) as ei:
        ib.step_periodic_noalloc(P, 0, n, n, buf.data_ptr(), buf.data_ptr(), 1.0)
    assert ei.value.code == ib.E_ARG
    assert n * n > ib.NOALLOC_MAX_CELLS
