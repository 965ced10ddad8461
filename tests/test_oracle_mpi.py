"""The reference's own shared-memory MPI mode through the one-node MPI
stand-in (oracle/mpi_shim): IB_RANKS=N forks N ranks that share the
reference's windows (DataArray.H:108-114, 415-446) and form its node layout
(mpiparams.cpp:68-105, SHN = N).

* the stand-in's self-check (oracle/mpi_shim/shim_check.cpp) passes for 1 to
  8 ranks, and an MPI_Abort or an early exit on one rank ends all of them;
* the reference's step run with several ranks leaves the same state as its
  one-rank run, cell for cell (keyed by level and position, since the
  reference orders its arrays by rank share): the periodic vortex and the
  static airfoil (3 levels, immersed body, wall forces) bit for bit, forces
  within a few ulps (the ranks' partial sums are added in rank order); the
  pitching airfoil across a regrid within 1e-15;
* the benchmark's reference arm runs this mode and reports its rank count.
"""
import io
import json
import os
import subprocess
import sys
import tempfile
from contextlib import redirect_stdout

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)
import bench  # noqa: E402
from pyoracle import read_dump  # noqa: E402

pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(REF, "shim_check")),
                                reason="reference oracle not built (make -C oracle)")


def run(args, ranks, env=None, timeout=300):
    e = dict(os.environ, IB_RANKS=str(ranks), IB_MPI_TIMEOUT="60", **(env or {}))
    return subprocess.run(args, env=e, capture_output=True, text=True, timeout=timeout)


@pytest.mark.parametrize("ranks", [1, 2, 3, 8])
def test_shim_self_check(ranks):
    r = run([os.path.join(REF, "shim_check")], ranks)
    assert r.returncode == 0, r.stderr
    assert f"SHIM_OK ranks={ranks}" in r.stdout


@pytest.mark.parametrize("mode,code", [("abort", 7), ("exit", 97)])
def test_one_failing_rank_ends_the_node(mode, code):
    r = run([os.path.join(REF, "shim_check"), mode], 4, timeout=120)
    assert r.returncode == code
    assert "SHIM_OK" not in r.stdout


def states(binary, env, ranks, step):
    with tempfile.TemporaryDirectory() as wd:
        e = dict(env, IB_DUMP=os.path.join(wd, "st"), IB_DUMP_AT=str(step), IB_STEPS=str(step),
                 IB_FORCE_LOG=os.path.join(wd, "f.bin"))
        r = subprocess.run([os.path.join(REF, binary)], cwd=wd, capture_output=True, text=True,
                           env=dict(os.environ, IB_RANKS=str(ranks), IB_MPI_TIMEOUT="120", **e),
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        res = next(json.loads(l.split(" ", 1)[1]) for l in r.stdout.splitlines()
                   if l.startswith("ORACLE_RESULT"))
        assert res["ranks"] == ranks
        d = read_dump(os.path.join(wd, f"st_{step:06d}.bin"))
        forces = np.fromfile(os.path.join(wd, "f.bin"))
    key = np.stack([d["level"], d["ix"], d["iy"]], axis=1)
    order = np.lexsort((key[:, 2], key[:, 1], key[:, 0]))
    return key[order], d["kind"][order], d["prim"].reshape(-1, 7)[order], forces


CASES = {
    "vortex": ("ref_vortex_vanleer", {"IB_NX": "64", "IB_STAGES": "4"}, 4, 3),
    "naca": ("ref_naca_minmod", {"IB_NX": "64", "IB_LEVELS": "3", "IB_STAGES": "4",
                                 "IB_USER_INIT": "0", "IB_FORCES": "1", "IB_NPTS": "120"}, 6, 4),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_several_ranks_leave_the_one_rank_state(name):
    binary, env, step, ranks = CASES[name]
    k1, kind1, p1, f1 = states(binary, env, 1, step)
    kn, kindn, pn, fn = states(binary, env, ranks, step)
    assert np.array_equal(k1, kn) and np.array_equal(kind1, kindn)
    assert np.array_equal(p1, pn), f"{np.count_nonzero(np.any(p1 != pn, axis=1))} cells differ"
    assert f1.shape == fn.shape
    scale = max(np.abs(f1).max(), 1.0)
    assert np.abs(f1 - fn).max() <= 1e-14 * scale


def test_moving_body_with_a_regrid_under_several_ranks():
    """The pitching airfoil across a regrid (step 20): the same mesh and the
    same state but for a few cells whose image-point values the ranks sum in
    another order (within 1e-15 relative)."""
    env = {"IB_NX": "64", "IB_LEVELS": "4", "IB_STAGES": "4", "IB_USER_INIT": "0",
           "IB_FORCES": "1", "IB_NPTS": "150", "IB_REGRID_EVERY": "20", "IB_PITCH_K": "2.0"}
    k1, kind1, p1, f1 = states("ref_pitch_minmod", env, 1, 24)
    kn, kindn, pn, fn = states("ref_pitch_minmod", env, 4, 24)
    assert np.array_equal(k1, kn) and np.array_equal(kind1, kindn)
    scale = np.abs(p1).max(axis=0)
    scale[scale == 0] = 1.0
    assert (np.abs(p1 - pn) / scale).max() <= 1e-15
    assert np.abs(f1 - fn).max() <= 1e-14 * max(np.abs(f1).max(), 1.0)


def test_reference_arm_runs_the_mpi_mode(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    monkeypatch.setattr(bench, "host_cores", lambda: 3)

    class Args:
        gpus, steps, warmup, n = 1, 2, 3, 64
    out = io.StringIO()
    with redirect_stdout(out):
        assert bench.reference_arm(Args()) == 0
    r = json.loads(out.getvalue().strip())
    assert r["cpu_baseline"]["cores"] == 3 and r["cpu_baseline"]["kind"] == "reference"
    assert r["config"]["same_config"] is True and r["config"]["grid_run"] == "64x64"
    assert "3 MPI ranks" in r["config"]["parallelism"]
    assert r["value"] > 0 and r["steps"] == 2


def test_reference_grid_shrinks_to_the_host_memory(monkeypatch):
    monkeypatch.setattr(bench, "avail_bytes", lambda: 1e12)
    assert bench.reference_grid(2048, 16) == 2048
    monkeypatch.setattr(bench, "avail_bytes", lambda: 20e9)
    assert bench.reference_grid(2048, 16) == 1024
