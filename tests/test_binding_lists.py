"""The reference-side C++ binding (immsered-boundary_b200/binding/
ibgpu_ns_solver.H) compiled into the reference solver (no GPU): from the
reference's own NACA0012 mesh and state it hands the C ABI exactly the cell
list, flags, state rows, coarse/fine pairs, domain ghosts, immersed-boundary
records and case constants that the GPU parity tests upload from the
reference's dump of the same run (workloads.naca_lists / naca_params)."""
import ctypes
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from conftest import ORACLE_DIR, load_pkg

sys.path.insert(0, ORACLE_DIR)
import pyoracle  # noqa: E402

BINARY = os.path.join(ORACLE_DIR, "_ref", "ref_naca_minmod_binding")
CASE_ENV = {"IB_NX": "64", "IB_LEVELS": "3", "IB_STAGES": "4", "IB_USER_INIT": "0",
            "IB_NPTS": "120", "IB_STEPS": "0"}

pytestmark = pytest.mark.skipif(not os.path.exists(BINARY),
                                reason="binding oracle not built (make -C oracle)")


def run_binding():
    work = tempfile.mkdtemp(prefix="binding_")
    env = dict(os.environ, **CASE_ENV, IB_DUMP=os.path.join(work, "d"),
               IB_BINDING_LISTS=os.path.join(work, "lists.bin"))
    out = subprocess.run([BINARY], cwd=work, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    d = pyoracle.read_dump(os.path.join(work, "d_000000.bin"))
    d["prim"] = d["prim"].reshape(1, -1, 7)
    d["scalars"] = d["scalars"].reshape(1, -1)
    return d, pyoracle.read_dump(os.path.join(work, "lists.bin"))


def test_binding_hands_the_abi_the_dumped_lists():
    pkg = load_pkg()
    ib, wl = pkg.ibgpu, pkg.workloads
    d, b = run_binding()
    want = wl.naca_lists(d, 0)
    for k in ("level", "ix", "iy", "flags"):
        assert np.array_equal(b[k], want[k]), k
    assert np.array_equal(b["prim"].reshape(-1, 7), want["prim"])
    for k, w in (("res", 11), ("pro", 11), ("bc", 7), ("ib", 18), ("patch", 17)):
        assert np.array_equal(b[k].reshape(-1, w), want[k]), k
    for k, w in (("bc_nmv", 3), ("facevar", 7), ("ib_f", 16), ("patch_f", 19),
                 ("body_center", 3)):
        assert np.array_equal(b[k].reshape(-1, w), want[k]), k
    assert np.array_equal(b["bc_scalars"], want["bc_scalars"])
    # the mesh is a real AMR mesh with a body: every list is populated
    assert all(len(want[k]) for k in ("res", "pro", "bc", "ib", "patch"))
    # case constants: the same bytes as the parity tests' ibgpu_case
    case = ib.make_case(wl.naca_params(d, 0, ib.FP64))
    assert b["case"].tobytes() == bytes(case)
    assert ctypes.sizeof(case) == 4 * len(b["case"])


def test_binding_context_creation_status():
    import torch
    _, b = run_binding()
    rc = int(b["create_rc"][0])
    if torch.cuda.is_available():
        assert rc == 0
    else:
        assert rc == load_pkg().ibgpu.E_CUDA  # reported, not aborted


def _forces(binary, extra):
    work = tempfile.mkdtemp(prefix="binding_run_")
    log = os.path.join(work, "forces.bin")
    env = dict(os.environ, **{**CASE_ENV, "IB_STEPS": "20", "IB_FORCES": "1",
                              "IB_FORCE_LOG": log, **extra})
    out = subprocess.run([binary], cwd=work, env=env, capture_output=True, text=True, timeout=300)
    return out, (np.fromfile(log, np.float64) if os.path.exists(log) else None)


def test_binding_build_keeps_the_reference_step():
    """Without IB_BINDING_STEP the binding build runs the reference's own step:
    its force history equals the plain reference build's bit for bit."""
    out, with_binding = _forces(BINARY, {})
    assert out.returncode == 0, out.stderr[-2000:]
    out, plain = _forces(os.path.join(ORACLE_DIR, "_ref", "ref_naca_minmod"), {})
    assert out.returncode == 0, out.stderr[-2000:]
    assert len(plain) > 0 and np.array_equal(with_binding, plain)


def test_binding_step_without_gpu_reports_the_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the binding step would run")
    out, _ = _forces(BINARY, {"IB_BINDING_STEP": "1"})
    assert out.returncode == 3 and "ibgpu_create" in out.stderr


def test_binding_cells_of_the_periodic_vortex():
    """Single periodic level: block (periodic) ghosts become alias rows, the
    cell list and flags equal the ones the vortex parity tests upload."""
    pkg = load_pkg()
    ib = pkg.ibgpu
    binary = os.path.join(ORACLE_DIR, "_ref", "ref_vortex_vanleer_binding")
    work = tempfile.mkdtemp(prefix="binding_vortex_")
    env = dict(os.environ, IB_NX="32", IB_STAGES="4", IB_STEPS="0",
               IB_DUMP=os.path.join(work, "d"), IB_BINDING_LISTS=os.path.join(work, "lists.bin"))
    out = subprocess.run([binary], cwd=work, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    d = pyoracle.read_dump(os.path.join(work, "d_000000.bin"))
    b = pyoracle.read_dump(os.path.join(work, "lists.bin"))
    flags = ib.cell_flags_from_boxes(d["kind"], d["solid"], d["infect"], d["signdis"], False)
    for k in ("level", "ix", "iy"):
        assert np.array_equal(b[k], d[k]), k
    assert np.array_equal(b["flags"], flags)
    assert np.array_equal(b["prim"], d["prim"])
    alias = (b["flags"] & ib.CELL_ALIAS) != 0
    assert alias.sum() == (32 + 4) ** 2 - 32 * 32  # the two-cell periodic frame
    assert len(b["res"]) == len(b["pro"]) == len(b["ib"]) == 0


def test_binding_tag_boxes_are_the_ones_tagthebox_judges():
    """The boxes the binding's TagLevel hands ibgpu_tag_plain / _learned are
    those the case's AMR::TagtheBox judges on the finished mesh (its tag
    dump, pass 1): same order, positions, centres and wall distances."""
    work = tempfile.mkdtemp(prefix="binding_tags_")
    env = dict(os.environ, **CASE_ENV, IB_TAG_DUMP=os.path.join(work, "tags.bin"),
               IB_BINDING_LISTS=os.path.join(work, "lists.bin"))
    out = subprocess.run([BINARY], cwd=work, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    rows = np.fromfile(os.path.join(work, "tags.bin"), np.float64).reshape(-1, 9)
    rows = rows[rows[:, 8] == 1]
    b = pyoracle.read_dump(os.path.join(work, "lists.bin"))
    assert len(rows) == len(b["tag_level"]) > 0
    for col, k in enumerate(("tag_level", "tag_ix", "tag_iy")):
        assert np.array_equal(rows[:, col].astype(np.int32), b[k]), k
    for col, k in ((3, "tag_xc"), (4, "tag_yc"), (5, "tag_signdis")):
        assert np.array_equal(rows[:, col], b[k]), k


def test_binding_tag_rule_takes_each_levels_requests():
    """TagLevel hands the GPU the case's regions with the requests the
    regrid made of that level (AMRLevel::torefine / toderefine), not the
    rule's own: for every level and every request (refine only, coarsen
    only, both) the plain criterion with the binding's level rule reproduces
    the case's AMR::TagtheBox decisions box for box, although the case rule
    it starts from requests both on every level."""
    pkg = load_pkg()
    ib, wl = pkg.ibgpu, pkg.workloads
    import indicator_oracle as io
    work = tempfile.mkdtemp(prefix="binding_tagcheck_")
    nlev = int(CASE_ENV["IB_LEVELS"])
    env = dict(os.environ, **CASE_ENV, IB_DUMP=os.path.join(work, "d"),
               IB_BINDING_TAGCHECK=work)
    # the base rule: every level asks for both (what a rule built once holds)
    out = subprocess.run([BINARY], cwd=work, env=dict(env, IB_BINDING_TAGCHECK=""),
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    d0 = pyoracle.read_dump(os.path.join(work, "d_000000.bin"))
    dh = d0["dh"].reshape(-1, 3)[:, 0]
    base = wl.naca_tag_rule(nlev, dh)
    assert base["torefine"][:nlev].all() and base["toderefine"][1:nlev].all()
    with open(os.path.join(work, "rule.bin"), "wb") as f:
        f.write(bytes(ib.make_tag_rule(base)))
    out = subprocess.run([BINARY], cwd=work, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    rows = np.fromfile(os.path.join(work, "tags.bin"), np.float64).reshape(-1, 9)
    lr = pyoracle.read_dump(os.path.join(work, "levelrule.bin"))["levelrule"].reshape(-1, 4)
    assert len(lr) == 3 * nlev
    req = {0: (1, 0), 1: (0, 1), 2: (1, 1)}
    changed = 0
    for pas, level, tor, toder in lr:
        assert (tor, toder) == req[(pas - 2) % 3], (pas, level, tor, toder)
        r = rows[rows[:, 8] == pas]
        if len(r):
            want = io.tags_from_rftag(r[:, 6], r[:, 7])
        else:  # TagtheBox returned before its loops: every box keeps
            r = rows[rows[:, 8] == 2 + 3 * level]
            want = np.zeros(len(r), np.uint8)
        assert len(r) and np.all(r[:, 0] == level)
        rule = {k: (np.array(v) if isinstance(v, np.ndarray) else v) for k, v in base.items()}
        rule["torefine"] = base["torefine"].copy()
        rule["toderefine"] = base["toderefine"].copy()
        rule["torefine"][level] = tor
        rule["toderefine"][level] = toder
        got = io.tag_plain(rule, r[:, 0].astype(int), r[:, 3], r[:, 4], r[:, 5])
        assert np.array_equal(got, want), (pas, level, int(np.sum(got != want)))
        # the base rule alone would have decided differently wherever the
        # request withholds refinement or coarsening
        changed += int(np.sum(io.tag_plain(base, r[:, 0].astype(int), r[:, 3], r[:, 4],
                                           r[:, 5]) != want))
    assert changed > 0


def test_binding_build_keeps_the_reference_moving_step():
    """The moving-body build with the binding linked in but not stepping on
    the GPU runs the reference's own moving step: the force history equals
    the plain reference build's bit for bit."""
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    outs = []
    for b in ("ref_pitch_minmod_binding", "ref_pitch_minmod"):
        work = tempfile.mkdtemp(prefix="pitch_")
        log = os.path.join(work, "forces.bin")
        env = dict(os.environ)
        env.update(make_golden.PITCH_ENV)
        env.update(IB_STEPS="25", IB_FORCE_LOG=log)
        out = subprocess.run([os.path.join(ORACLE_DIR, "_ref", b)], cwd=work, env=env,
                             capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr[-2000:]
        outs.append(np.fromfile(log, np.float64))
    assert len(outs[0]) == 25 * 15 and np.array_equal(outs[0], outs[1])
    # and it is the recorded moving-body history
    ref = make_golden.load("pitch_forces_s100_n64_l4")["history"][:25].ravel()
    assert np.array_equal(outs[1], ref)
