"""GPU step parity on the static NACA0012 AMR case (3 levels, immersed body,
far-field boundaries, viscous, subcycling) against the reference solver's
own dumps (tests/golden/naca_minmod_s4_n64_l3.npz).

Covers restriction and prolongation on their schedules, the domain ghosts
(pressure inlet/outlet, outflow copy), the immersed-boundary ghost cells,
the frozen viscous flux, the subcycled stage updates of each level and the
wall forces, step by step from the reference's own state.
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

NAME = "naca_minmod_s4_n64_l3"
REL_FP64 = 1e-12
REL_MIXED = 5e-5
FORCE_TOL = 1e-3  # |dCl|, |dCd| bar of the airfoil workloads


def naca_solver(ib, g, k, precision):
    return workloads.naca_solver(g, k, precision)


def conserved(prim):
    r, u, v, e = prim[:, 0], prim[:, 1], prim[:, 2], prim[:, 6]
    return np.stack([r, r * u, r * v, r * e], axis=1)


def rel_err(got, ref):
    cg, cr = conserved(got), conserved(ref)
    scale = np.abs(cr).max(axis=0)
    scale[scale == 0] = 1.0
    return (np.abs(cg - cr).max(axis=0) / scale).max()


def describe_mismatch(g, got, ref, mask):
    bad = mask & np.any(got != ref, axis=1)
    out = []
    for l in np.unique(g["level"][bad]):
        m = bad & (g["level"] == l)
        kinds = {int(k): int(np.sum(m & (g["kind"] == k))) for k in np.unique(g["kind"][m])}
        out.append(f"level {l}: {int(m.sum())} rows {kinds}")
    return "; ".join(out)


def test_exact_build_matches_reference_each_step(cuda_lib, pkg):
    ib = pkg.ibgpu
    g = make_golden.load(NAME)
    rows = np.ones(len(g["level"]), bool)
    for k in range(g["prim"].shape[0] - 1):
        sol = naca_solver(ib, g, k, ib.FP64_EXACT)
        d = sol.time_marching(k)
        assert d.abort_code == 0
        assert sol.dt == g["scalars"][k + 1][1]
        got = sol.download()
        ref = g["prim"][k + 1]
        # viscosity goes through pow(T, 3) and the inlet through pow(x, 3.5):
        # correctly rounded here, libm-rounded in the reference
        err = rel_err(got, ref)
        assert err <= 1e-15, f"step {k}: rel err {err:.3e}: {describe_mismatch(g, got, ref, rows)}"
        f = sol.wall_forces().ravel()
        assert np.allclose(f, g["forces"][k + 1], rtol=1e-13, atol=1e-15), (f, g["forces"][k + 1])
        sol.close()


def test_fp64_build_within_1e12_each_step(cuda_lib, pkg):
    ib = pkg.ibgpu
    g = make_golden.load(NAME)
    for k in range(g["prim"].shape[0] - 1):
        sol = naca_solver(ib, g, k, ib.FP64)
        sol.time_marching(k)
        got = sol.download()
        assert rel_err(got, g["prim"][k + 1]) <= REL_FP64
        sol.close()


def test_mixed_build_and_forces_within_tolerance(cuda_lib, pkg):
    ib = pkg.ibgpu
    g = make_golden.load(NAME)
    sol = naca_solver(ib, g, 0, ib.MIXED)
    for k in range(g["prim"].shape[0] - 1):
        sol.time_marching(k)
    got = sol.download()
    assert rel_err(got, g["prim"][-1]) <= REL_MIXED
    f = sol.wall_forces()
    ref = g["forces"][-1].reshape(-1, 6)
    # lift/drag coefficients with F_ref = 0.5 rho u^2 * chord * slab depth
    F_ref = 0.5 * 1.0 * 0.1
    assert np.abs(f[:, :2] - ref[:, :2]).max() / F_ref < FORCE_TOL
    sol.close()


def test_four_steps_in_a_row_match_reference(cuda_lib, pkg):
    """Subcycling over a full coarse-level period: the GPU keeps the state
    and runs the four steps itself."""
    ib = pkg.ibgpu
    g = make_golden.load(NAME)
    sol = naca_solver(ib, g, 0, ib.FP64)
    for k in range(g["prim"].shape[0] - 1):
        d = sol.time_marching(k)
        assert d.abort_code == 0
    got = sol.download()
    assert rel_err(got, g["prim"][-1]) <= 4 * REL_FP64
    f = sol.wall_forces().ravel()
    assert np.allclose(f, g["forces"][-1], rtol=1e-10, atol=1e-13)
    sol.close()


def force_history():
    with np.load(os.path.join(os.path.dirname(__file__), "golden",
                              "naca_forces_s400_n64_l3.npz")) as z:
        return z["history"]


@pytest.mark.parametrize("precision,tol_coef,dt_rtol", [
    ("exact", 1e-12, 1e-12), ("fp64", 1e-10, 1e-10), ("mixed", FORCE_TOL, 1e-4)])
def test_cl_cd_history_matches_reference(cuda_lib, pkg, precision, tol_coef, dt_rtol):
    """400 steps from the reference's initial state: the drag/lift history
    (force_foil.dat columns Fx/F_ref, Fy/F_ref) and the dt history against
    the reference's own run, step by step."""
    ib = pkg.ibgpu
    prec = {"exact": ib.FP64_EXACT, "fp64": ib.FP64, "mixed": ib.MIXED}[precision]
    g = make_golden.load(NAME)
    hist = force_history()
    F_ref = 0.5 * 1.0 * 0.1
    sol = naca_solver(ib, g, 0, prec)
    worst = np.zeros(2)
    for k in range(len(hist)):
        d = sol.time_marching(k)
        assert d.abort_code == 0
        assert abs(sol.dt - hist[k, 2]) <= dt_rtol * hist[k, 2]
        f = sol.wall_forces()[0]
        coef = np.abs(f[:2] - hist[k, 3:5]) / F_ref
        worst = np.maximum(worst, coef)
    print(f"\n{precision}: max |dCd| {worst[0]:.2e}, max |dCl| {worst[1]:.2e} over {len(hist)} steps")
    assert worst.max() <= tol_coef
    sol.close()
