"""The learned refinement indicator deciding the runtime regrids of the
reference solver's own NACA0012 run, and the drag/lift deviation that
results.

The reference's host regrid (AMR::PerformAdaptive, run every 2 steps with
refinement and coarsening requested on every level) asks a tag server for
each level's decisions (oracle/cases/case_naca.cpp, IB_TAG_SERVER).  The
server here builds the GPU solver from the state the reference dumps just
before the regrid and answers with the MLP's decisions (ibgpu_tag_learned:
features and BF16 tensor-core inference on the device), except on every
10th regrid, where the plain criterion decides (the deployment policy); on
those the GPU's plain criterion (ibgpu_tag_plain) must equal the reference's
own decision box for box, on meshes that earlier learned regrids shaped.
The flow between regrids is the reference's FP64 step.  The plain
criterion alone never changes this static-airfoil mesh, so its run is the
reference's run without regrids; the learned run's Cl/Cd history is held
against it.
"""
import os
import subprocess
import sys
import tempfile
import time

import numpy as np
import pytest

from conftest import GOLDEN_DIR, ORACLE_DIR, load_pkg

sys.path.insert(0, ORACLE_DIR)
sys.path.insert(0, GOLDEN_DIR)
import make_golden  # noqa: E402
import pyoracle  # noqa: E402

pytestmark = pytest.mark.gpu

pkg = load_pkg()
ib, wl, ind = pkg.ibgpu, pkg.workloads, pkg.indicator
NAME = "naca_minmod_s4_n64_l3"
BINARY = os.path.join(ORACLE_DIR, "_ref", "ref_naca_minmod")
BINARY_TRAIN = os.path.join(ORACLE_DIR, "_ref", "ref_naca_vanleer")
CASE_ENV = {"IB_NX": "64", "IB_LEVELS": "3", "IB_STAGES": "4", "IB_USER_INIT": "0",
            "IB_FORCES": "1", "IB_NPTS": "120"}
STEPS = 400
REGRID_EVERY = 2
JUDGE_EVERY = 10
F_REF = 0.5 * 1.0 * 0.1  # force scale of the Cl/Cd coefficients (force_foil.dat)
CL_CD_TOL = 1e-3         # |dCl|, |dCd| bar of the airfoil workloads


def trained_indicator(runtime_rule):
    """MLP trained on the plain criterion's decisions: for the record's boxes
    while the mesh is built and re-judged (both tag passes, features from
    four states of a GPU run), and at every 10th runtime regrid of the
    reference's run with the other limiter (VanLeer; the deployment run uses
    minmod), features from the GPU solver holding that run's state."""
    import torch
    g = make_golden.load(NAME)
    with np.load(os.path.join(GOLDEN_DIR, NAME + ".npz")) as z:
        t, dh = z["tags"], z["dh"].reshape(-1, 3)[:, 0]
    key = t[:, 0] * 1e8 + t[:, 1] * 1e4 + t[:, 2]
    _, first = np.unique(key, return_index=True)
    t = t[np.sort(first)]
    mesh = set(zip(g["level"].tolist(), g["ix"].tolist(), g["iy"].tolist()))
    t = t[[(int(a), int(b), int(c)) in mesh for a, b, c in t[:, :3]]]
    B = dict(level=t[:, 0].astype(np.int32), ix=t[:, 1].astype(np.int32),
             iy=t[:, 2].astype(np.int32), xc=t[:, 3], yc=t[:, 4], signdis=t[:, 5])
    sol = wl.naca_solver(g, 0, ib.FP64)
    rule = wl.naca_tag_rule(3, dh)
    gen_labels = ind.classes_from_tags(sol.tag_plain(rule, B["level"], B["xc"], B["yc"],
                                                     B["signdis"]))
    li = ind.LearnedIndicator(sol, seed=0)
    feats, labels = [], []
    for s in range(4):
        feats.append(li.features(rule, B))
        labels.append(gen_labels)
        sol.run(2 * s, 2)

    def collect(work, ts, level, rows):
        plain = rows[:, 6].astype(np.int32)
        if (ts // REGRID_EVERY - 1) % JUDGE_EVERY == 0:
            st = state_solver(os.path.join(work, f"state_{ts}.bin"))
            li.solver = st
            feats.append(li.features(runtime_rule, boxes_of(rows)))
            labels.append(class_of_decision(plain))
            st.close()
        return plain

    run_reference(collect, BINARY_TRAIN)
    li.solver = sol
    li.train(torch.cat(feats).contiguous(), np.concatenate(labels), steps=800, batch=4096,
             lr=3e-3)
    return li, sol


def state_solver(path):
    """GPU solver holding the mesh and state of a reference dump."""
    d = pyoracle.read_dump(path)
    d["prim"] = d["prim"].reshape(1, -1, 7)
    d["scalars"] = d["scalars"].reshape(1, -1)
    return wl.naca_solver(d, 0, ib.FP64)


def boxes_of(rows):
    return dict(level=rows[:, 0].astype(np.int32), ix=rows[:, 1].astype(np.int32),
                iy=rows[:, 2].astype(np.int32), xc=rows[:, 3], yc=rows[:, 4], signdis=rows[:, 5])


def class_of_decision(dec):
    """The case's decision code -> the indicator's classes."""
    dec = np.asarray(dec)
    return np.where(dec == 1, ind.CLASS_REFINE,
                    np.where(dec == 2, ind.CLASS_COARSEN, ind.CLASS_KEEP)).astype(np.uint8)


def decision_of_tags(bits):
    """IBGPU_TAG_* bits -> the case's decision code (0 keep, 1 refine, 2 coarsen)."""
    bits = np.asarray(bits)
    return np.where(bits & ib.TAG_REFINE, 1, np.where(bits & ib.TAG_COARSEN, 2, 0)).astype(np.int32)


def run_reference(server=None, binary=BINARY):
    """The reference's run with regrids every REGRID_EVERY steps; with a
    server, its decisions answer each level's request.  Returns the force
    history (per step ts, t, dt, 6 per body) and the ORACLE_REGRID lines."""
    work = tempfile.mkdtemp(prefix="regrid_")
    env = dict(os.environ, **CASE_ENV, IB_STEPS=str(STEPS), IB_REGRID_EVERY=str(REGRID_EVERY),
               IB_FORCE_LOG=os.path.join(work, "forces.bin"))
    if server is not None:
        env["IB_TAG_SERVER"] = work
    # the reference's output goes to a file: a pipe nobody reads while the
    # server loop runs would fill and stall it
    log = open(os.path.join(work, "out.txt"), "w")
    proc = subprocess.Popen([binary], cwd=work, env=env, stdout=log, stderr=subprocess.STDOUT)
    deadline = time.monotonic() + 600
    try:
        done = set()
        while server is not None:
            assert time.monotonic() < deadline, "reference run did not finish"
            reqs = sorted(f for f in os.listdir(work)
                          if f.startswith("req_") and f.endswith(".bin") and f not in done)
            if not reqs:
                if proc.poll() is not None:
                    break
                time.sleep(0.002)
                continue
            for f in reqs:
                ts, level = (int(x) for x in f[4:-4].split("_"))
                rows = np.fromfile(os.path.join(work, f), np.float64).reshape(-1, 7)
                dec = np.ascontiguousarray(server(work, ts, level, rows), np.int32)
                tmp = os.path.join(work, "tmp_" + f)
                dec.tofile(tmp)
                os.rename(tmp, os.path.join(work, "resp_" + f[4:]))
                done.add(f)
        proc.wait(timeout=max(1.0, deadline - time.monotonic()))
    finally:
        if proc.poll() is None:
            proc.kill()
            proc.wait()
        log.close()
    with open(os.path.join(work, "out.txt")) as f:
        out = f.read()
    assert proc.returncode == 0, out[-2000:]
    hist = np.fromfile(os.path.join(work, "forces.bin"), np.float64).reshape(STEPS, -1)
    return hist, [l.split()[1:] for l in out.splitlines() if l.startswith("ORACLE_REGRID")]


def total_force(hist):
    """(Fx, Fy) summed over the bodies (upper and lower surface) per step."""
    nb = (hist.shape[1] - 3) // 6
    return sum(hist[:, 3 + 6 * b:5 + 6 * b] for b in range(nb))


def test_learned_regrids_cl_cd_deviation(cuda_lib):
    g = make_golden.load(NAME)
    rule = wl.naca_tag_rule(3, g["dh"].reshape(-1, 3)[:, 0])
    # runtime regrids request refinement below the finest level only (the
    # reference's AMR::CheckLevelRefineFlag) and coarsening above level 0
    rule = dict(rule, torefine=rule["torefine"].copy())
    rule["torefine"][2] = 0
    li, train_sol = trained_indicator(rule)
    plain_hist, _ = run_reference()
    # plain regrids leave the mesh as built: the run is the reference's run
    # without regrids (its committed 400-step force history), bit for bit
    with np.load(os.path.join(GOLDEN_DIR, "naca_forces_s400_n64_l3.npz")) as z:
        assert np.array_equal(plain_hist, z["history"][:STEPS])
    state = {"ts": None, "sol": None}
    judged = []  # (ts, level, fraction of boxes whose learned decision differs)
    applied = []  # learned decisions served

    def server(work, ts, level, rows):
        if state["ts"] != ts:
            if state["sol"] is not None:
                state["sol"].close()
            state["sol"] = state_solver(os.path.join(work, f"state_{ts}.bin"))
            state["ts"] = ts
        li.solver = state["sol"]
        B = boxes_of(rows)
        learned = decision_of_tags(li.tags(rule, B))
        regrid = ts // REGRID_EVERY - 1
        if regrid % JUDGE_EVERY:
            applied.extend(learned.tolist())
        if regrid % JUDGE_EVERY == 0:
            plain = decision_of_tags(state["sol"].tag_plain(rule, B["level"], B["xc"], B["yc"],
                                                            B["signdis"], B["ix"], B["iy"]))
            # the GPU's plain criterion equals the reference's decision
            assert np.array_equal(plain, rows[:, 6].astype(np.int32)), (ts, level)
            judged.append((ts, level, float(np.mean(learned != plain))))
            return plain
        return learned

    try:
        learned_hist, regrids = run_reference(server)
    finally:
        if state["sol"] is not None:
            state["sol"].close()
        train_sol.close()
    assert len(regrids) == 3 * (STEPS // REGRID_EVERY)
    boxes = sum(int(r[2]) for r in regrids)
    differ = sum(int(r[3]) for r in regrids)
    kept = sum(int(r[4]) for r in regrids)
    dF = np.abs(total_force(learned_hist) - total_force(plain_hist)) / F_REF
    d_cd, d_cl = dF.max(axis=0)
    mis = np.mean([j[2] for j in judged])
    first = [int(r[2]) for r in regrids[:3]]
    last = [int(r[2]) for r in regrids[-3:]]
    print(f"\nleaf boxes per level at the first / last regrid: {first} / {last}; learned "
          f"decisions by class (keep, refine, coarsen): {np.bincount(applied, minlength=3)}")
    print(f"\n{len(regrids) // 3} regrids over {STEPS} steps: learned decisions differing from "
          f"the plain ones {differ / boxes:.4f} of {boxes} box decisions (mismatch at the judged "
          f"regrids {mis:.4f}), {kept} inadmissible decisions kept; max |dCd| {d_cd:.2e}, "
          f"max |dCl| {d_cl:.2e}")
    assert np.allclose(learned_hist[:, 2], plain_hist[:, 2], rtol=0.05)  # dt history
    assert d_cd < CL_CD_TOL and d_cl < CL_CD_TOL
