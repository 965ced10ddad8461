"""The allocation-free step entry point (ibgpu_step_periodic_noalloc).

Callers that may not allocate device memory while they run (a coupler whose
device memory belongs to another framework, a time loop that cannot take
cudaMalloc's device-wide synchronisation) hand the library their own device
buffers; everything else lives in the library's fixed device array.  Here the
test plays that caller: torch owns the in/out buffers, the library allocates
nothing, and two consecutive steps must agree with the regular entry point
(ibgpu_step through a context) within the FP64 parity tolerance.

Kept in a file of its own that sorts last, so a run that stops at the first
failure has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_FP64 = 1e-12


def test_noalloc_step_matches_regular_entry_point_twice(cuda_lib, pkg):
    import torch

    ib, wl = pkg.ibgpu, pkg.workloads
    n = 64
    P, cells, prim = wl.vortex_case(n, nstages=4, precision=ib.FP64)

    # regular entry point: context, uploads, two steps
    sol = ib.FlowSolver(P)
    sol.upload_topology(**cells)
    sol.init_flow(prim)
    ref = []
    for ts in range(2):
        sol.time_marching(ts)
        ref.append((sol.download(), sol.dt))
    sol.close()

    # allocation-free entry point on caller-owned device rows (row-major cells)
    rows = torch.from_numpy(prim).to("cuda")
    out = torch.empty_like(rows)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    dt = P["dt0"]
    src = rows
    for ts in range(2):
        dt, diag = ib.step_periodic_noalloc(P, ts, n, n, src.data_ptr(), out.data_ptr(), dt, stream)
        assert diag.abort_code == 0 and diag.cells_marched == n * n
        got = out.cpu().numpy()
        want, want_dt = ref[ts]
        assert dt == want_dt
        scale = np.abs(want).max(axis=0)
        scale[scale == 0] = 1.0
        assert (np.abs(got - want).max(axis=0) / scale).max() <= REL_FP64
        src = out  # second call steps in place, continuing from the first


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
