"""Regenerate the golden fixtures from the reference solver itself.

Runs the reference-solver oracle binaries (built from the reference's own
sources by ``make -C oracle``) on small cases and packs their state dumps
into compressed .npz files next to this script.  The fixtures pin both the
C restatement of the step (oracle/ib_oracle.c) and the GPU path.

    make -C oracle REF=<reference dir> && python tests/golden/make_golden.py

Each fixture holds the box list of the z = 0 plane (level, ix, iy, kind,
ptype, solid, infect, signdis), the case constants, and the primitive state
(roe, u, v, w, p, T, e) plus scalars (t, dt, CFL_dt, ts, ...) of every dumped
step.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")

# the plain-method airfoil workload at its stated size
CONFIG1_ENV = {"IB_NX": "128", "IB_LEVELS": "4", "IB_STAGES": "4", "IB_USER_INIT": "0",
               "IB_FORCES": "1", "IB_NPTS": "200"}

# the moving-body workload at a test size: the pitching NACA0015 (Mach 0.2,
# Re 1e4, [0,30]^2) on a 64^2 base grid + 3 AMR levels, 150 points per
# surface, regrids every 20 steps, pitching at reduced frequency 2 (omega 4)
# so that the body moves across cells within the recorded steps
PITCH_ENV = {"IB_NX": "64", "IB_LEVELS": "4", "IB_STAGES": "4", "IB_USER_INIT": "0",
             "IB_FORCES": "1", "IB_NPTS": "150", "IB_REGRID_EVERY": "20", "IB_PITCH_K": "2.0"}

# name -> (binary, environment, number of steps)
CASES = {
    "vortex_vanleer_s4_n32": ("ref_vortex_vanleer", {"IB_NX": "32", "IB_STAGES": "4"}, 4),
    "vortex_minmod_s3_n32": ("ref_vortex_minmod", {"IB_NX": "32", "IB_STAGES": "3"}, 3),
    # static NACA0012, 3 levels, immersed body, far-field boundaries, Re 5000:
    # covers restriction/prolongation schedules, boundary ghosts, IB cells,
    # viscous fluxes, subcycling and the wall forces
    "naca_minmod_s4_n64_l3": ("ref_naca_minmod", {"IB_NX": "64", "IB_LEVELS": "3",
                                                  "IB_STAGES": "4", "IB_USER_INIT": "0",
                                                  "IB_FORCES": "1", "IB_NPTS": "120"}, 4),
    # the plain-method airfoil workload at its stated size: 128^2 base + 3 AMR
    # levels (~45k leaf cells), 400-point NACA0012, Mach 0.5, 2 deg, Re 5000,
    # minmod, 4 stages, CFL 0.5: the mesh, the initial state and two steps
    "naca_minmod_s4_n128_l4": ("ref_naca_minmod", CONFIG1_ENV, 2),
    # the reference's other domain boundary conditions (BCValues.H:191-298) on
    # the 3-level airfoil mesh: fixed values / fixed velocity / slip wall /
    # no-slip wall, and pressure inlet / outlet / static-frame wall / slip wall
    "naca_bc_a_s4_n64_l3": ("ref_naca_minmod", {"IB_NX": "64", "IB_LEVELS": "3",
                                                "IB_STAGES": "4", "IB_USER_INIT": "0",
                                                "IB_FORCES": "1", "IB_NPTS": "120",
                                                "IB_BC": "-10,-45,-51,-49"}, 4),
    "naca_bc_b_s4_n64_l3": ("ref_naca_minmod", {"IB_NX": "64", "IB_LEVELS": "3",
                                                "IB_STAGES": "4", "IB_USER_INIT": "0",
                                                "IB_FORCES": "1", "IB_NPTS": "120",
                                                "IB_BC": "-13,-12,-46,-51"}, 4),
}
# plain tag criterion only (TagtheBox on the initial mesh, refine and coarsen
# requested on every level): name -> (binary, environment)
TAG_CASES = {
    "naca_tags_n64_l4": ("ref_naca_minmod", {"IB_NX": "64", "IB_LEVELS": "4", "IB_USER_INIT": "0",
                                             "IB_NPTS": "200"}),
}
# force histories (Cl/Cd time series) of longer runs of a case above, started
# from that case's initial state: name -> (binary, environment, steps)
FORCE_CASES = {
    "naca_forces_s400_n64_l3": ("ref_naca_minmod", {"IB_NX": "64", "IB_LEVELS": "3",
                                                   "IB_STAGES": "4", "IB_USER_INIT": "0",
                                                   "IB_FORCES": "1", "IB_NPTS": "120"}, 400),
    # the stated 1000 steps of the plain-method airfoil workload
    "naca_forces_s1000_n128_l4": ("ref_naca_minmod", CONFIG1_ENV, 1000),
    # the moving body: 100 steps, four regrids
    "pitch_forces_s100_n64_l4": ("ref_pitch_minmod", PITCH_ENV, 100),
}
# states of a developed flow, too large to commit (about 1 MB each): the
# fixture records the SHA-256 of each dumped state's bytes and its scalars,
# and live_states() regenerates them with the same binary and checks the
# digests: name -> (binary, environment, dumped step counts)
STATE_DIGEST_CASES = {
    "naca_states_s600_n128_l4": ("ref_naca_minmod", CONFIG1_ENV, (600, 601, 602, 603, 604)),
    # the moving body: states and moved lists around steps where cells enter
    # or leave the body (22, 23, 50, 58), after the regrids at 20 and 40
    "pitch_states_n64_l4": ("ref_pitch_minmod", PITCH_ENV, (21, 22, 23, 49, 50, 57, 58)),
}
# per-case records that do not change between dumps of a static mesh
AUX = ("cf_res", "cf_pro", "bc", "bc_nmv", "facevar", "bc_scalars", "ib", "ib_f", "patch",
       "patch_f", "body_f")

STATIC = ("level", "ix", "iy", "kind", "ptype", "solid", "infect", "signdis")


def run_case(name: str, binary: str, env: dict, steps: int) -> str:
    work = tempfile.mkdtemp(prefix="golden_")
    try:
        e = dict(os.environ)
        e.update(env)
        e["IB_STEPS"] = str(steps)
        e["IB_DUMP"] = os.path.join(work, "d")
        if "IB_BC" not in env:
            e["IB_TAG_DUMP"] = os.path.join(work, "tags.bin")
        subprocess.run([os.path.join(REF, binary)], cwd=work, env=e, check=True,
                       stdout=subprocess.DEVNULL)
        snaps = [pyoracle.read_dump(os.path.join(work, f"d_{k:06d}.bin")) for k in range(steps + 1)]
        out = {k: snaps[0][k] for k in STATIC}
        for k in ("dh", "schedule", "initvar", "domain") + AUX:
            if k in snaps[0]:
                out[k] = snaps[0][k]
        for s in snaps[1:]:
            for k in STATIC:
                if not np.array_equal(s[k], snaps[0][k]):
                    raise RuntimeError(f"{name}: topology changed between dumps ({k})")
        out["prim"] = np.stack([s["prim"].reshape(-1, 7) for s in snaps])
        out["scalars"] = np.stack([s["scalars"] for s in snaps])
        # wall forces exist after each step (none for the initial state)
        nf = max(len(s["forces"]) for s in snaps)
        out["forces"] = np.stack([s["forces"] if len(s["forces"]) == nf else np.full(nf, np.nan)
                                  for s in snaps])
        tpath = os.path.join(work, "tags.bin")
        tags = np.fromfile(tpath, dtype=np.float64).reshape(-1, 9) if os.path.exists(tpath) else []
        if len(tags):
            out["tags"] = tags
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        return path
    finally:
        shutil.rmtree(work, ignore_errors=True)


def run_tag_case(name: str, binary: str, env: dict) -> str:
    """(level, ix, iy, centre x, centre y, signdis, tag, detag, pass) of every
    normal box, as the case's AMR::TagtheBox leaves them after its loops:
    pass 0 while the mesh is built, pass 1 re-judging the finished mesh."""
    work = tempfile.mkdtemp(prefix="golden_")
    try:
        e = dict(os.environ)
        e.update(env)
        e["IB_STEPS"] = "0"
        e["IB_DUMP"] = os.path.join(work, "d")
        e["IB_TAG_DUMP"] = os.path.join(work, "tags.bin")
        subprocess.run([os.path.join(REF, binary)], cwd=work, env=e, check=True,
                       stdout=subprocess.DEVNULL)
        tags = np.fromfile(os.path.join(work, "tags.bin"), dtype=np.float64).reshape(-1, 9)
        dh = pyoracle.read_dump(os.path.join(work, "d_000000.bin"))["dh"]
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, tags=tags, dh=dh)
        return path
    finally:
        shutil.rmtree(work, ignore_errors=True)


def load(name: str) -> dict:
    with np.load(os.path.join(HERE, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def snapshot(g: dict, k: int) -> dict:
    """Dump-shaped dict of snapshot k (what pyoracle.OracleLevels expects)."""
    d = {key: g[key] for key in STATIC + ("dh", "schedule", "initvar", "domain") + AUX if key in g}
    d["prim"] = g["prim"][k].ravel()
    d["scalars"] = g["scalars"][k]
    return d


def run_force_case(name: str, binary: str, env: dict, steps: int) -> str:
    """ts, t, dt and each body's force and moment after every step."""
    work = tempfile.mkdtemp(prefix="golden_")
    try:
        e = dict(os.environ)
        e.update(env)
        e["IB_STEPS"] = str(steps)
        e["IB_FORCE_LOG"] = os.path.join(work, "forces.bin")
        subprocess.run([os.path.join(REF, binary)], cwd=work, env=e, check=True,
                       stdout=subprocess.DEVNULL)
        hist = np.fromfile(os.path.join(work, "forces.bin"), dtype=np.float64).reshape(steps, -1)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, history=hist)
        return path
    finally:
        shutil.rmtree(work, ignore_errors=True)


def _dump_states(binary: str, env: dict, at, work: str) -> list:
    e = dict(os.environ)
    e.update(env)
    e["IB_STEPS"] = str(max(at))
    e["IB_DUMP"] = os.path.join(work, "d")
    e["IB_DUMP_AT"] = ",".join(str(k) for k in (0,) + tuple(at))
    subprocess.run([os.path.join(REF, binary)], cwd=work, env=e, check=True,
                   stdout=subprocess.DEVNULL)
    return [pyoracle.read_dump(os.path.join(work, f"d_{k:06d}.bin")) for k in (0,) + tuple(at)]


def _digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_state_digest_case(name: str, binary: str, env: dict, at) -> str:
    """SHA-256 of the prim rows of every dumped step, and its scalars."""
    work = tempfile.mkdtemp(prefix="golden_")
    try:
        snaps = _dump_states(binary, env, at, work)[1:]
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, steps=np.array(at, np.int64),
                            digests=np.array([_digest(s["prim"]) for s in snaps]),
                            scalars=np.stack([s["scalars"] for s in snaps]))
        return path
    finally:
        shutil.rmtree(work, ignore_errors=True)


def live_snapshots(name: str) -> list:
    """The dumps a STATE_DIGEST_CASES fixture records, regenerated by its
    reference binary and checked against the recorded digests: one complete
    dump per recorded step (mesh lists, flags, immersed-boundary records and
    state), for runs whose mesh or body moves between dumps."""
    binary, env, at = STATE_DIGEST_CASES[name]
    rec = load(name)
    work = tempfile.mkdtemp(prefix="live_")
    try:
        snaps = _dump_states(binary, env, at, work)[1:]
    finally:
        shutil.rmtree(work, ignore_errors=True)
    for s, want, k in zip(snaps, rec["digests"], at):
        if _digest(s["prim"]) != str(want):
            raise RuntimeError(f"{name}: the live reference run differs from the recorded one "
                               f"at step {k}")
        s["step"] = k
    return snaps


def record_of(snap: dict, state_from: dict | None = None) -> dict:
    """A single-snapshot record (the layout of ``load``) of one dump: its
    mesh and lists, with the state and scalars of ``state_from`` if given."""
    src = state_from if state_from is not None else snap
    out = {k: snap[k] for k in STATIC + ("dh", "schedule", "initvar", "domain") + AUX if k in snap}
    out["prim"] = src["prim"].reshape(1, -1, 7)
    out["scalars"] = src["scalars"].reshape(1, -1)
    return out


def live_states(name: str) -> dict:
    """The states a STATE_DIGEST_CASES fixture records, regenerated by its
    reference binary and checked against the recorded digests; returned in
    the layout of ``load`` (mesh lists, prim and scalars per dumped step)."""
    binary, env, at = STATE_DIGEST_CASES[name]
    rec = load(name)
    work = tempfile.mkdtemp(prefix="live_")
    try:
        snaps = _dump_states(binary, env, at, work)
    finally:
        shutil.rmtree(work, ignore_errors=True)
    for s, want, k in zip(snaps[1:], rec["digests"], at):
        if _digest(s["prim"]) != str(want):
            raise RuntimeError(f"{name}: the live reference run differs from the recorded one "
                               f"at step {k}")
    out = {k: snaps[0][k] for k in STATIC}
    for k in ("dh", "schedule", "initvar", "domain") + AUX:
        if k in snaps[0]:
            out[k] = snaps[0][k]
    out["prim"] = np.stack([s["prim"].reshape(-1, 7) for s in snaps[1:]])
    out["scalars"] = np.stack([s["scalars"] for s in snaps[1:]])
    out["forces"] = np.stack([s["forces"] for s in snaps[1:]])
    out["steps"] = np.array(at)
    return out


if __name__ == "__main__":
    names = sys.argv[1:] or (list(CASES) + list(TAG_CASES) + list(FORCE_CASES) +
                             list(STATE_DIGEST_CASES))
    for n in names:
        if n in STATE_DIGEST_CASES:
            print(run_state_digest_case(n, *STATE_DIGEST_CASES[n]))
        elif n in TAG_CASES:
            print(run_tag_case(n, *TAG_CASES[n]))
        elif n in FORCE_CASES:
            print(run_force_case(n, *FORCE_CASES[n]))
        else:
            b, env, steps = CASES[n]
            print(run_case(n, b, env, steps))
