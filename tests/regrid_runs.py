"""Reference runs whose regrids move the mesh (test helper): the NACA case
regridding every 2 steps with refinement and coarsening requested on every
level, a tag server answering with the plain criterion's decisions of which
a seeded random share is replaced (the case file keeps any decision its
regrid would reject), and a state dump after every regrid.  Used to test
lists that the reference rebuilds in its regrids against the reference's
own lists on meshes the plain criterion alone would never produce."""
import os
import subprocess
import tempfile
import time

import numpy as np

from conftest import ORACLE_DIR, load_oracle

BINARY = os.path.join(ORACLE_DIR, "_ref", "ref_naca_minmod")


def noisy_regrid_dumps(levels: int, seed: int, steps: int = 40, share: float = 0.05, nx: int = 64):
    """State dumps (pyoracle.read_dump dicts) after each of the run's
    steps // 2 regrids."""
    pyoracle = load_oracle()
    work = tempfile.mkdtemp(prefix="regrid_dumps_")
    env = dict(os.environ, IB_NX=str(nx), IB_LEVELS=str(levels), IB_STAGES="4",
               IB_USER_INIT="0", IB_NPTS="120", IB_STEPS=str(steps), IB_REGRID_EVERY="2",
               IB_DUMP_EVERY="2", IB_TAG_SERVER=work, IB_DUMP=os.path.join(work, "d"))
    rng = np.random.default_rng(seed)
    log = open(os.path.join(work, "out.txt"), "w")
    proc = subprocess.Popen([BINARY], cwd=work, env=env, stdout=log, stderr=subprocess.STDOUT)
    deadline = time.monotonic() + 600
    done = set()
    try:
        while True:
            assert time.monotonic() < deadline, "reference run timed out"
            reqs = sorted(f for f in os.listdir(work)
                          if f.startswith("req_") and f.endswith(".bin") and f not in done)
            if not reqs:
                if proc.poll() is not None:
                    break
                time.sleep(0.002)
                continue
            for f in reqs:
                rows = np.fromfile(os.path.join(work, f), np.float64).reshape(-1, 7)
                d = rows[:, 6].astype(np.int32).copy()
                flip = rng.random(len(d)) < share
                d[flip] = rng.integers(0, 3, int(flip.sum()))
                tmp = os.path.join(work, "tmp_" + f)
                d.tofile(tmp)
                os.rename(tmp, os.path.join(work, "resp_" + f[4:]))
                done.add(f)
    finally:
        if proc.poll() is None:
            proc.kill()
            proc.wait()
        log.close()
    assert proc.returncode == 0, open(os.path.join(work, "out.txt")).read()[-2000:]
    return [pyoracle.read_dump(os.path.join(work, f"d_{k:06d}.bin")) for k in range(2, steps + 1, 2)]
