"""The GPU list builder of the coarse/fine interfaces
(ibgpu_build_interfaces) against the reference's own lists: after every one
of 20 regrids of reference runs steered away from the plain criterion (3
and 4 levels; tests/regrid_runs.py), the restriction pairs with their
layers, the prolongation pairs and the interface ghost cells built on the
device from the leaf cells equal the reference's, row for row (both sorted
by level, y, x; the reference's repeated prolongation entries counted
once), and the same lists for the stated plain-method mesh."""
import ctypes
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402
from conftest import ORACLE_DIR, load_pkg  # noqa: E402
from regrid_runs import BINARY, noisy_regrid_dumps  # noqa: E402

sys.path.insert(0, ORACLE_DIR)
import interfaces_oracle as io  # noqa: E402

pytestmark = pytest.mark.gpu


def check(sol, d, nlev):
    leaf = d["kind"] == 0
    got = sol.build_interfaces(nlev, d["level"][leaf], d["ix"][leaf], d["iy"][leaf])
    want = io.reference_lists(d)
    for name, a, b in zip(("restriction", "prolongation", "ghost"), got, want):
        assert a.shape == b.shape and np.array_equal(a, b), name
    return [len(a) for a in got]


def test_interfaces_of_the_stated_airfoil_mesh(cuda_lib, pkg):
    ib, wl = pkg.ibgpu, pkg.workloads
    g = make_golden.load("naca_minmod_s4_n128_l4")
    P, cells, prim = wl.vortex_case(16)
    sol = ib.FlowSolver(P)  # any context: the builder needs a stream only
    n = check(sol, g, 4)
    assert min(n) > 0
    sol.close()


@pytest.mark.skipif(not os.path.exists(BINARY), reason="reference oracle not built")
@pytest.mark.parametrize("levels,seed", [(3, 7), (4, 11)])
def test_interfaces_after_reference_regrids(cuda_lib, pkg, levels, seed):
    ib, wl = pkg.ibgpu, pkg.workloads
    P, cells, prim = wl.vortex_case(16)
    sol = ib.FlowSolver(P)
    dumps = noisy_regrid_dumps(levels, seed)
    assert len(dumps) == 20
    for k, d in enumerate(dumps):
        check(sol, d, levels)
    # capacities below the counts: counts returned, nothing written
    leaf = dumps[0]["kind"] == 0
    cols = [np.ascontiguousarray(dumps[0][k][leaf], np.int32) for k in ("level", "ix", "iy")]
    i32 = ctypes.POINTER(ctypes.c_int32)
    cells = ib.Cells(int(leaf.sum()), *[c.ctypes.data_as(i32) for c in cols], None)
    out = ib.InterfaceLists()
    rc = ib.lib().ibgpu_build_interfaces(sol._ctx, levels, ctypes.byref(cells), ctypes.byref(out))
    assert rc == ib.E_ARG and out.nres > 0 and out.npro > 0 and out.nghost > 0
    sol.close()
