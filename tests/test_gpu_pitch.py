"""The moving immersed body: a NACA0015 pitching about its quarter chord
(Mach 0.2, Re 1e4, [0,30]^2), at a test size (64^2 base grid + 3 AMR
levels, 150 points per surface), pitching at reduced frequency 2 so that
the body crosses cells within the recorded steps, regrids every 20 steps.

The reference moves and re-immerses the body at the start of every step
(Body::IBConditions_Image -> MovingBody_Image, Body.cpp:1352-1357,
Bodymove.cpp:37-125): new wall distances, cells that leave or enter the
body, new immersed-boundary cells and image points, wall points moving with
the rotation (Body.H:709-721).  On the device the mesh and the state stay;
the new cell flags go through ibgpu_update_flags and the new
immersed-boundary records through ibgpu_upload_ib.

* per step, from the reference's own state with the lists the reference
  built for the next step, at steps where cells enter or leave the body
  (after the regrids at 20 and 40): exact build
  <= 1e-14, FP64 <= 1e-12, mixed <= 5e-5 relative on the conserved variables;
* the reference's own main loop stepping through the C++ binding on the
  device (GpuNS_Solver::MoveBodies + TimeMarching) for 100 steps and four
  regrids: the dt and force history against the reference's own run,
  exact <= 1e-12, FP64 <= 1e-10, mixed |dCl|, |dCd| < 1e-3;
* the same loop in the reference's shared-memory MPI mode (4 ranks, rank 0
  on the device): the 1-rank history.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402
from conftest import ORACLE_DIR, load_pkg  # noqa: E402

workloads = load_pkg().workloads

pytestmark = pytest.mark.gpu

STATES = "pitch_states_n64_l4"
HISTORY = "pitch_forces_s100_n64_l4"
BINARY = os.path.join(ORACLE_DIR, "_ref", "ref_pitch_minmod_binding")
REL = {"exact": 1e-14, "fp64": 1e-12, "mixed": 5e-5}
F_REF = 0.5 * 1.0 * 0.1


def conserved(prim):
    r, u, v, e = prim[:, 0], prim[:, 1], prim[:, 2], prim[:, 6]
    return np.stack([r, r * u, r * v, r * e], axis=1)


def rel_err(got, ref):
    cg, cr = conserved(got), conserved(ref)
    scale = np.abs(cr).max(axis=0)
    scale[scale == 0] = 1.0
    return (np.abs(cg - cr).max(axis=0) / scale).max()


def prec_of(ib, name):
    return {"exact": ib.FP64_EXACT, "fp64": ib.FP64, "mixed": ib.MIXED}[name]


@pytest.fixture(scope="module")
def snaps():
    return make_golden.live_snapshots(STATES)


def pairs(snaps):
    """(before, after) dumps of consecutive steps on the same mesh."""
    out = []
    for a, b in zip(snaps, snaps[1:]):
        if b["step"] == a["step"] + 1:
            assert all(np.array_equal(a[k], b[k]) for k in ("level", "ix", "iy", "kind"))
            out.append((a, b))
    return out


def test_the_body_moves_between_the_recorded_steps(snaps):
    for a, b in pairs(snaps):
        ia = set(map(tuple, a["ib"].reshape(-1, 20)[:, :2].tolist()))
        ib_ = set(map(tuple, b["ib"].reshape(-1, 20)[:, :2].tolist()))
        changed = len(ia ^ ib_) + int(np.sum(a["solid"] != b["solid"]))
        assert changed > 0, (a["step"], b["step"])  # cells enter or leave the body
        assert np.abs(b["ib_f"].reshape(-1, 16)[:, 13:16]).max() > 0.05  # wall velocity
    assert len(pairs(snaps)) == 4


@pytest.mark.parametrize("precision", ["exact", "fp64", "mixed"])
def test_step_with_the_moved_body_from_reference_states(cuda_lib, pkg, snaps, precision):
    """The device holds step k's mesh, lists and state; the body moves (new
    flags through ibgpu_update_flags, new records through ibgpu_upload_ib);
    one step; the reference's state after step k + 1."""
    ib = pkg.ibgpu
    for a, b in pairs(snaps):
        sol = workloads.naca_solver(make_golden.record_of(a), 0, prec_of(ib, precision))
        moved = workloads.naca_lists(make_golden.record_of(b, state_from=a), 0)
        sol.update_flags(moved["flags"])
        sol.upload_ib(moved["ib"], moved["ib_f"], moved["patch"], moved["patch_f"],
                      moved["body_center"])
        d = sol.time_marching(int(a["step"]))
        assert d.abort_code == 0
        if precision == "exact":
            assert sol.dt == b["scalars"][1]
        err = rel_err(sol.download(), b["prim"].reshape(-1, 7))
        assert err <= REL[precision], f"step {a['step']} -> {b['step']}: rel err {err:.3e}"
        f = sol.wall_forces().ravel()
        ftol = {"exact": 1e-12, "fp64": 1e-10, "mixed": 1e-4}[precision]
        assert np.allclose(f, b["forces"], rtol=ftol, atol=1e-14), precision
        sol.close()


def test_flag_update_keeps_the_layout(cuda_lib, pkg, snaps):
    """A flag update may not change which rows are leaf cells, present or
    periodic copies: that needs a topology upload."""
    ib = pkg.ibgpu
    a = snaps[0]
    sol = workloads.naca_solver(make_golden.record_of(a), 0, ib.FP64)
    flags = workloads.naca_lists(make_golden.record_of(a), 0)["flags"].copy()
    sol.update_flags(flags)  # unchanged: fine
    leaf = np.flatnonzero(flags & ib.CELL_NORMAL)[0]
    flags[leaf] = np.uint8(int(flags[leaf]) & ~ib.CELL_NORMAL & 0xFF)
    with pytest.raises(ib.IbgpuError) as ei:
        sol.update_flags(flags)
    assert ei.value.code == ib.E_TOPOLOGY
    # the refused update changed nothing on the device: a step there equals
    # a step of a context that never saw it
    sol.time_marching(int(a["step"]))
    ref = workloads.naca_solver(make_golden.record_of(a), 0, ib.FP64)
    ref.time_marching(int(a["step"]))
    assert np.array_equal(sol.download(), ref.download())
    ref.close()
    sol.close()


def test_flag_update_of_the_changed_rows_only(cuda_lib, pkg, snaps):
    """New flags for the rows whose flags a move changed (each of them
    sent twice) step the same bits as the full flag update; a row index out
    of range or a changed layout bit is refused and changes nothing."""
    ib = pkg.ibgpu
    a, b = pairs(snaps)[0]
    old = workloads.naca_lists(make_golden.record_of(a), 0)["flags"]
    moved = workloads.naca_lists(make_golden.record_of(b, state_from=a), 0)
    rows = np.flatnonzero(old != moved["flags"])
    assert len(rows) > 0
    out = []
    for full in (True, False):
        sol = workloads.naca_solver(make_golden.record_of(a), 0, ib.FP64)
        if full:
            sol.update_flags(moved["flags"])
        else:
            with pytest.raises(ib.IbgpuError) as e:
                sol.update_flags_rows([0, sol.ncells], moved["flags"][:2])
            assert e.value.code == ib.E_ARG
            leaf = int(np.flatnonzero(old & ib.CELL_NORMAL)[0])
            with pytest.raises(ib.IbgpuError) as e:
                sol.update_flags_rows([leaf], [int(old[leaf]) & ~ib.CELL_NORMAL & 0xFF])
            assert e.value.code == ib.E_TOPOLOGY
            twice = np.r_[rows, rows]
            sol.update_flags_rows(twice, moved["flags"][twice])
        sol.upload_ib(moved["ib"], moved["ib_f"], moved["patch"], moved["patch_f"],
                      moved["body_center"])
        sol.time_marching(int(a["step"]))
        out.append(sol.download())
        sol.close()
    assert np.array_equal(out[0], out[1])


def run_binding(precision, steps=100, ranks=1):
    work = tempfile.mkdtemp(prefix="pitch_binding_")
    log = os.path.join(work, "forces.bin")
    env = dict(os.environ)
    env.update(make_golden.PITCH_ENV)
    env.update(IB_STEPS=str(steps), IB_FORCE_LOG=log, IB_BINDING_STEP="1", IB_RANKS=str(ranks),
               IB_MPI_TIMEOUT="300",
               IB_BINDING_PRECISION=str({"fp64": 0, "exact": 1, "mixed": 2}[precision]))
    out = subprocess.run([BINARY], cwd=work, env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    return np.fromfile(log, np.float64).reshape(steps, -1), out.stdout


@pytest.mark.skipif(not os.path.exists(BINARY), reason="binding oracle not built (make -C oracle)")
@pytest.mark.parametrize("precision,tol", [("exact", 1e-12), ("fp64", 1e-10), ("mixed", 1e-3)])
def test_reference_loop_moves_the_body_through_the_binding(cuda_lib, precision, tol):
    ref = make_golden.load(HISTORY)["history"]
    got, _ = run_binding(precision)
    assert got.shape == ref.shape and np.array_equal(got[:, 0], ref[:, 0])
    dt_err = np.abs(got[:, 2] - ref[:, 2]) / ref[:, 2]
    fg = got[:, 3:].reshape(len(ref), -1, 6)[:, :, :2]
    fr = ref[:, 3:].reshape(len(ref), -1, 6)[:, :, :2]
    coef = np.abs(fg - fr).max() / F_REF
    total = np.abs(fg.sum(axis=1) - fr.sum(axis=1)).max() / F_REF
    print(f"\npitching {precision}: max rel dt {dt_err.max():.2e}, max |dC| per surface "
          f"{coef:.2e}, airfoil {total:.2e}")
    assert coef <= tol and total <= tol
    assert dt_err.max() <= (tol if precision != "mixed" else 1e-4)


@pytest.mark.skipif(not os.path.exists(BINARY), reason="binding oracle not built (make -C oracle)")
def test_binding_in_the_references_mpi_mode(cuda_lib):
    """The same loop with the reference's host code on 4 ranks of one
    shared-memory node (rank 0 drives the device, every rank re-immerses
    its share of the moving body and regrids): the 1-rank binding's dt and
    force history, to the reference's own rank-count dependence (partial
    sums added in rank order)."""
    one, _ = run_binding("fp64", steps=30)
    four, out = run_binding("fp64", steps=30, ranks=4)
    assert '"ranks": 4' in out
    assert one.shape == four.shape and np.array_equal(one[:, 0], four[:, 0])
    assert np.abs(one[:, 2] - four[:, 2]).max() <= 1e-12 * np.abs(one[:, 2]).max()
    f1, f4 = one[:, 3:], four[:, 3:]
    assert np.abs(f1 - f4).max() <= 1e-10 * F_REF


@pytest.mark.skipif(not os.path.exists(BINARY), reason="binding oracle not built (make -C oracle)")
@pytest.mark.parametrize("ranks", [1, 4])
def test_device_wall_distances_equal_the_references_passes(cuda_lib, ranks):
    """Every step of 25 (a regrid at 20) the device wall-distance passes
    (ibgpu_wall_distance) from the same pairs as the reference's own
    RenewLevelDistance and SynNormal_BlockDistance: every box's pair and
    solid flag bit for bit and the move lists entry for entry, on each rank's
    share."""
    env = dict(os.environ)
    env.update(make_golden.PITCH_ENV)
    work = tempfile.mkdtemp(prefix="pitch_distcheck_")
    env.update(IB_STEPS="25", IB_BINDING_STEP="1", IB_BINDING_DISTCHECK="1",
               IB_RANKS=str(ranks), IB_MPI_TIMEOUT="300")
    out = subprocess.run([BINARY], cwd=work, env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    res = next(json.loads(l.split(" ", 1)[1]) for l in out.stdout.splitlines()
               if l.startswith("ORACLE_RESULT"))
    assert res["ranks"] == ranks
    assert res["move_phases_seconds"]["distcheck_mismatches"] == 0
