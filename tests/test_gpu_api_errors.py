"""Error behaviour of the newer C-ABI entry points on a GPU: empty inputs
are accepted, inconsistent ones rejected with IBGPU_E_ARG / IBGPU_E_STATE,
and the context stays usable afterwards."""
import numpy as np
import pytest

from conftest import load_pkg

pytestmark = pytest.mark.gpu

pkg = load_pkg()
ib, wl = pkg.ibgpu, pkg.workloads


def vortex_solver(n=32, precision=ib.FP64, **kw):
    P, cells, prim = wl.vortex_case(n, precision=precision, **kw)
    s = ib.FlowSolver(P)
    s.upload_topology(**cells)
    s.init_flow(prim)
    return s


def test_tag_entry_points_reject_bad_input(cuda_lib):
    s = vortex_solver()
    rule = wl.naca_tag_rule(1, [10.0 / 32])
    empty = np.zeros(0, np.int32)
    assert len(s.tag_plain(rule, empty, np.zeros(0), np.zeros(0), np.zeros(0))) == 0
    with pytest.raises(ib.IbgpuError) as e:
        s.tag_plain(rule, np.array([99], np.int32), np.zeros(1), np.zeros(1), np.zeros(1))
    assert e.value.code == ib.E_ARG
    # a box that is not a cell of the uploaded mesh (a level it does not
    # have) has no stencil
    import torch
    feat = torch.empty((1, ib.MLP_IN), dtype=torch.int16, device="cuda")
    with pytest.raises(ib.IbgpuError) as e:
        s.indicator_features(rule, np.array([3], np.int32), np.array([0], np.int32),
                             np.array([0], np.int32), np.zeros(1), np.zeros(1), np.zeros(1),
                             feat.data_ptr())
    assert e.value.code == ib.E_ARG
    # still usable
    d = s.time_marching(0)
    assert d.abort_code == 0
    s.close()


def test_mlp_rejects_misaligned_features(cuda_lib):
    import torch
    s = vortex_solver()
    P = torch.from_numpy(pkg.indicator.init_params(0)).cuda()
    X = torch.zeros((3, ib.MLP_IN + 1), dtype=torch.int16, device="cuda")
    cls = torch.empty(2, dtype=torch.uint8, device="cuda")
    with pytest.raises(ib.IbgpuError) as e:
        s.mlp_forward(P.data_ptr(), 2, X.data_ptr() + 2, cls.data_ptr())  # 2-byte offset
    assert e.value.code == ib.E_ARG
    s.close()


def test_batch_rejects_mismatched_cases(cuda_lib):
    a = vortex_solver(precision=ib.FP64)
    b = vortex_solver(precision=ib.MIXED)
    c = vortex_solver(precision=ib.FP64_EXACT)
    for group in ([a, b], [c]):
        with pytest.raises(ib.IbgpuError) as e:
            ib.Batch(group)
        assert e.value.code == ib.E_ARG
    for s in (a, b, c):
        s.close()


def test_state_calls_before_upload(cuda_lib):
    P, cells, prim = wl.vortex_case(32)
    s = ib.FlowSolver(P)
    with pytest.raises(ib.IbgpuError) as e:
        s.upload_signdis(np.zeros(len(prim)))
    assert e.value.code == ib.E_STATE
    s.upload_topology(**cells)
    with pytest.raises(ib.IbgpuError) as e:
        s.time_marching(0)
    assert e.value.code == ib.E_STATE
    with pytest.raises(ib.IbgpuError) as e:
        s.step_async(0)
    assert e.value.code == ib.E_STATE
    s.close()


def test_pipelined_entry_points_reject_bad_input(cuda_lib):
    s = vortex_solver()
    with pytest.raises(ib.IbgpuError) as e:
        s.step_result()  # no chain open
    assert e.value.code == ib.E_STATE
    s.dt = 0.0  # a chain must start from a positive dt
    with pytest.raises(ib.IbgpuError) as e:
        s.step_async(0)
    assert e.value.code == ib.E_ARG
    s.dt = 1.0
    with pytest.raises(ib.IbgpuError) as e:
        s.step_async(-1)
    assert e.value.code == ib.E_ARG
    s.step_async(0)
    # a new mesh ends the chain; the context stays usable
    P, cells, prim = wl.vortex_case(32)
    s.upload_topology(**cells)
    s.init_flow(prim)
    with pytest.raises(ib.IbgpuError) as e:
        s.step_result()
    assert e.value.code == ib.E_STATE
    d = s.time_marching(0)
    assert d.abort_code == 0
    s.close()
