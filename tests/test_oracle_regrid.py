"""The reference's runtime regrids as the learned-regrid measurement uses them
(no GPU): the NACA case regridding every 2 steps with refinement and
coarsening requested decides exactly as without regrids when the plain
criterion decides, whether the case decides itself or a tag server echoes
its plain decisions back; and a server answering with noisy decisions runs
through, its inadmissible decisions kept as boxes instead of aborting the
reference (oracle/cases/case_naca.cpp, IB_REGRID_EVERY / IB_TAG_SERVER)."""
import os
import subprocess
import tempfile
import time

import numpy as np
import pytest

from conftest import ORACLE_DIR

BINARY = os.path.join(ORACLE_DIR, "_ref", "ref_naca_minmod")
CASE_ENV = {"IB_NX": "64", "IB_LEVELS": "3", "IB_STAGES": "4", "IB_USER_INIT": "0",
            "IB_FORCES": "1", "IB_NPTS": "120"}
STEPS = 20

pytestmark = pytest.mark.skipif(not os.path.exists(BINARY),
                                reason="reference oracle not built (make -C oracle)")


def run(extra, server=None):
    work = tempfile.mkdtemp(prefix="regrid_cpu_")
    env = dict(os.environ, **CASE_ENV, **extra, IB_STEPS=str(STEPS),
               IB_FORCE_LOG=os.path.join(work, "forces.bin"))
    if server is not None:
        env["IB_TAG_SERVER"] = work
    log = open(os.path.join(work, "out.txt"), "w")
    proc = subprocess.Popen([BINARY], cwd=work, env=env, stdout=log, stderr=subprocess.STDOUT)
    deadline = time.monotonic() + 300
    try:
        done = set()
        while server is not None:
            assert time.monotonic() < deadline
            reqs = sorted(f for f in os.listdir(work)
                          if f.startswith("req_") and f.endswith(".bin") and f not in done)
            if not reqs:
                if proc.poll() is not None:
                    break
                time.sleep(0.002)
                continue
            for f in reqs:
                rows = np.fromfile(os.path.join(work, f), np.float64).reshape(-1, 7)
                tmp = os.path.join(work, "tmp_" + f)
                np.ascontiguousarray(server(rows), np.int32).tofile(tmp)
                os.rename(tmp, os.path.join(work, "resp_" + f[4:]))
                done.add(f)
        proc.wait(timeout=max(1.0, deadline - time.monotonic()))
    finally:
        if proc.poll() is None:
            proc.kill()
            proc.wait()
        log.close()
    out = open(os.path.join(work, "out.txt")).read()
    assert proc.returncode == 0, out[-2000:]
    hist = np.fromfile(os.path.join(work, "forces.bin"), np.float64).reshape(STEPS, -1)
    return hist, [[int(x) for x in l.split()[1:]] for l in out.splitlines()
                  if l.startswith("ORACLE_REGRID")]


def test_plain_regrids_leave_the_run_unchanged():
    base, _ = run({})
    plain, _ = run({"IB_REGRID_EVERY": "2"})
    echoed, lines = run({"IB_REGRID_EVERY": "2"}, server=lambda r: r[:, 6])
    assert np.array_equal(plain, base)
    assert np.array_equal(echoed, base)
    assert len(lines) == 3 * (STEPS // 2)
    assert all(l[3] == 0 and l[4] == 0 for l in lines)  # nothing differs, nothing kept


def test_noisy_decisions_are_made_admissible():
    rng = np.random.default_rng(7)

    def noisy(rows):
        d = rows[:, 6].astype(np.int32).copy()
        flip = rng.random(len(d)) < 0.02
        d[flip] = rng.integers(0, 3, int(flip.sum()))
        return d

    hist, lines = run({"IB_REGRID_EVERY": "2"}, server=noisy)
    assert np.all(np.isfinite(hist))
    assert sum(l[3] for l in lines) > 0  # the mesh was steered away from the plain one
    assert sum(l[4] for l in lines) > 0  # and some decisions had to be kept
