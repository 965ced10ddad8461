"""The reference's other domain boundary conditions (BCValues::BCBoxTreat and
SetBCType_*, BCValues.H:51-298) on the 3-level NACA0012 mesh, against the
reference's own runs with those face types (tests/golden/naca_bc_*):

* a: fixed values (-10) at the inlet side, fixed velocity with zero-gradient
  pressure (-45) at the outlet side, slip wall (-51, normal of the reference
  cell's face) at the bottom, no-slip wall (-49) at the top;
* b: pressure inlet (-13), pressure outlet (-12), no-slip wall of a static
  frame (-46) at the bottom, slip wall at the top.

Per step from the reference's state: the exact build gives the domain ghost
cells bit for bit and every conserved variable within 1e-15 relative; the
FP64 build within 1e-12.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402
from conftest import load_pkg  # noqa: E402

workloads = load_pkg().workloads

CASES = {"naca_bc_a_s4_n64_l3": (-10, -45, -51, -49), "naca_bc_b_s4_n64_l3": (-13, -12, -46, -51)}
REL = {"exact": 1e-15, "fp64": 1e-12}


def conserved(prim):
    r, u, v, e = prim[:, 0], prim[:, 1], prim[:, 2], prim[:, 6]
    return np.stack([r, r * u, r * v, r * e], axis=1)


def rel_err(got, ref):
    cg, cr = conserved(got), conserved(ref)
    scale = np.abs(cr).max(axis=0)
    scale[scale == 0] = 1.0
    return (np.abs(cg - cr).max(axis=0) / scale).max()


@pytest.mark.parametrize("name", sorted(CASES))
def test_records_hold_the_boundary_types(name):
    g = make_golden.load(name)
    bc = g["bc"].reshape(-1, 9)
    inplane = bc[(bc[:, 7] == 0) & (bc[:, 8] == 0)]
    assert set(np.unique(inplane[:, 6]).tolist()) == set(CASES[name])
    nmv = g["bc_nmv"].reshape(-1, 3)[(bc[:, 7] == 0) & (bc[:, 8] == 0)]
    slip = inplane[:, 6] == -51
    assert slip.any() and np.all(np.abs(nmv[slip]).sum(axis=1) > 0)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["exact", "fp64"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_boundary_types_match_reference_each_step(cuda_lib, pkg, name, precision):
    ib = pkg.ibgpu
    g = make_golden.load(name)
    ghost = g["kind"] == 1  # domain ghost rows of the z = 0 plane
    prec = ib.FP64_EXACT if precision == "exact" else ib.FP64
    for k in range(g["prim"].shape[0] - 1):
        sol = workloads.naca_solver(g, k, prec)
        assert sol.time_marching(k).abort_code == 0
        got = sol.download()
        ref = g["prim"][k + 1]
        if precision == "exact":
            assert sol.dt == g["scalars"][k + 1][1]
            bad = np.flatnonzero(np.any(got[ghost] != ref[ghost], axis=1))
            assert len(bad) == 0, f"step {k}: {len(bad)} domain ghosts differ"
        err = rel_err(got, ref)
        assert err <= REL[precision], f"step {k}: rel err {err:.3e}"
        sol.close()
