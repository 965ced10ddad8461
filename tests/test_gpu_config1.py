"""The plain-method airfoil workload at its stated size against the
reference's own run: a 128 x 128 base grid on [0,20]^2 plus 3 AMR levels
around a 400-point NACA0012 (45,448 leaf cells), Mach 0.5, 2 degrees, Re 5000,
minmod MUSCL, all-speed Roe, 4 stages, CFL 0.5, 1000 steps, FP64.

* the first two steps from the reference's initial state (committed dumps);
* per-step parity over half a coarse-level period of the developed flow
  (steps 600 -> 604): the reference regenerates those states here and their
  committed SHA-256 digests pin them to the recorded run;
* the 1000-step drag/lift and dt history of the reference's run, step by step.

Tolerances: exact build <= 1e-15 relative per step on the conserved
variables (libm pow in the reference's viscosity and inlet terms against the
correctly rounded powers of the exact build), FP64 build <= 1e-12 per step
(the parity bar), mixed <= 5e-5 per step and |dCl|, |dCd| < 1e-3 over the
history (the accuracy gate of the airfoil workloads).
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402
from conftest import load_pkg  # noqa: E402

workloads = load_pkg().workloads

pytestmark = pytest.mark.gpu

NAME = "naca_minmod_s4_n128_l4"
STATES = "naca_states_s600_n128_l4"
HISTORY = "naca_forces_s1000_n128_l4"
REL = {"exact": 1e-15, "fp64": 1e-12, "mixed": 5e-5}
F_REF = 0.5 * 1.0 * 0.1  # 0.5 rho_inf u_inf^2 * chord * slab depth
COEF_TOL = {"exact": 1e-12, "fp64": 1e-10, "mixed": 1e-3}


def precision_of(ib, name):
    return {"exact": ib.FP64_EXACT, "fp64": ib.FP64, "mixed": ib.MIXED}[name]


def conserved(prim):
    r, u, v, e = prim[:, 0], prim[:, 1], prim[:, 2], prim[:, 6]
    return np.stack([r, r * u, r * v, r * e], axis=1)


def rel_err(got, ref):
    cg, cr = conserved(got), conserved(ref)
    scale = np.abs(cr).max(axis=0)
    scale[scale == 0] = 1.0
    return (np.abs(cg - cr).max(axis=0) / scale).max()


@pytest.fixture(scope="module")
def developed():
    # the reference's own run to step 604 on this host (about 20 s)
    return make_golden.live_states(STATES)


def test_workload_is_the_stated_size():
    g = make_golden.load(NAME)
    normal = g["kind"] == 0
    assert int(g["domain"][0]) == int(g["domain"][1]) == 128 and int(g["domain"][5]) == 4
    assert int(normal.sum()) == 45448
    assert len(g["patch"]) // 17 == 398  # 2 x 200 surface points -> 2 x 199 patches
    s = g["scalars"][0]
    assert s[8] == 0.5 and s[9] == 5000.0 and s[13] == 0.5 and int(s[14]) == 4


@pytest.mark.parametrize("precision", ["exact", "fp64", "mixed"])
def test_first_steps_match_reference(cuda_lib, pkg, precision):
    ib = pkg.ibgpu
    g = make_golden.load(NAME)
    for k in range(g["prim"].shape[0] - 1):
        sol = workloads.naca_solver(g, k, precision_of(ib, precision))
        d = sol.time_marching(k)
        assert d.abort_code == 0
        if precision == "exact":
            assert sol.dt == g["scalars"][k + 1][1]
        err = rel_err(sol.download(), g["prim"][k + 1])
        assert err <= REL[precision], f"step {k}: rel err {err:.3e}"
        f = sol.wall_forces().ravel()
        ftol = {"exact": 1e-13, "fp64": 1e-10, "mixed": 1e-4}[precision]
        assert np.allclose(f, g["forces"][k + 1], rtol=ftol, atol=1e-15), precision
        sol.close()


@pytest.mark.parametrize("precision", ["exact", "fp64", "mixed"])
def test_developed_flow_each_step(cuda_lib, pkg, developed, precision):
    """Steps 600 -> 604 (level 0 marches at 600, level 1 at 600 and 604,
    level 2 on the even steps, level 3 every step) from the reference's own
    states, one step at a time."""
    ib = pkg.ibgpu
    g = developed
    steps = g["steps"]
    for k in range(len(steps) - 1):
        sol = workloads.naca_solver(g, k, precision_of(ib, precision))
        d = sol.time_marching(int(steps[k]))
        assert d.abort_code == 0
        if precision == "exact":
            assert sol.dt == g["scalars"][k + 1][1]
        err = rel_err(sol.download(), g["prim"][k + 1])
        assert err <= REL[precision], f"step {steps[k]}: rel err {err:.3e}"
        sol.close()


def test_developed_flow_four_steps_on_the_device(cuda_lib, pkg, developed):
    ib = pkg.ibgpu
    g = developed
    sol = workloads.naca_solver(g, 0, ib.FP64)
    for k in range(len(g["steps"]) - 1):
        assert sol.time_marching(int(g["steps"][k])).abort_code == 0
    err = rel_err(sol.download(), g["prim"][-1])
    assert err <= 4 * REL["fp64"], f"rel err {err:.3e}"
    f = sol.wall_forces().ravel()
    assert np.allclose(f, g["forces"][-1], rtol=1e-10, atol=1e-13)
    sol.close()


def cl_cd(forces):
    """(Cd, Cl) of the airfoil: both surfaces' force, x and y components,
    over F_ref."""
    f = np.asarray(forces).reshape(-1, 6)
    return f[:, :2].sum(axis=0) / F_REF


@pytest.mark.parametrize("precision", ["exact", "fp64", "mixed"])
def test_cl_cd_history_1000_steps(cuda_lib, pkg, precision):
    """The stated 1000 steps from the reference's initial state: dt, the
    drag and lift of each surface and of the airfoil, step by step."""
    ib = pkg.ibgpu
    g = make_golden.load(NAME)
    hist = make_golden.load(HISTORY)["history"]
    assert hist.shape == (1000, 15)
    sol = workloads.naca_solver(g, 0, precision_of(ib, precision))
    worst = np.zeros(2)
    worst_body = 0.0
    dt_rtol = {"exact": 1e-12, "fp64": 1e-10, "mixed": 1e-4}[precision]
    for k in range(len(hist)):
        d = sol.time_marching(k)
        assert d.abort_code == 0
        assert abs(sol.dt - hist[k, 2]) <= dt_rtol * hist[k, 2], k
        f = sol.wall_forces()
        worst = np.maximum(worst, np.abs(cl_cd(f) - cl_cd(hist[k, 3:])))
        worst_body = max(worst_body, np.abs(f[:, :2] - hist[k, 3:].reshape(-1, 6)[:, :2]).max()
                         / F_REF)
    print(f"\n{precision}: max |dCd| {worst[0]:.2e}, max |dCl| {worst[1]:.2e}, per surface "
          f"{worst_body:.2e} over {len(hist)} steps")
    assert worst.max() <= COEF_TOL[precision] and worst_body <= COEF_TOL[precision]
    sol.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_one_case_batch_equals_run(cuda_lib, pkg, precision):
    """The graph-replayed batch entry point with this one case gives the bits
    of ibgpu_run over three coarse-level periods (24 steps: every level's
    schedule, the CFL passes and the folded CFL bound)."""
    ib = pkg.ibgpu
    g = make_golden.load(NAME)
    period = int(g["schedule"].reshape(-1, 6)[:, 0].max())
    steps = 3 * period
    ref = workloads.naca_solver(g, 0, precision_of(ib, precision))
    ref.run(0, steps)
    sol = workloads.naca_solver(g, 0, precision_of(ib, precision))
    b = ib.Batch([sol])
    d = b.run(0, steps)
    assert d[0].abort_code == 0
    assert sol.dt == ref.dt
    assert np.array_equal(sol.download(), ref.download())
    assert np.array_equal(sol.wall_forces(), ref.wall_forces())
    b.close()
    sol.close()
    ref.close()
