"""The oracle's case file for families of airfoil cases (no GPU): Mach
number, Reynolds number, angle of attack and thickness from the environment
reach the reference's gas constants and free stream (they are initialised
before FlowConstants.cpp derives its constants), and the seeded batched
airfoil cases of the benchmark span the stated ranges."""
import math
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from conftest import ORACLE_DIR, ROOT

sys.path.insert(0, ORACLE_DIR)
sys.path.insert(0, ROOT)
import pyoracle  # noqa: E402

BINARY = os.path.join(ORACLE_DIR, "_ref", "ref_naca_minmod")


@pytest.mark.skipif(not os.path.exists(BINARY), reason="reference oracle not built")
def test_case_constants_follow_the_environment():
    work = tempfile.mkdtemp(prefix="case_env_")
    env = dict(os.environ, IB_MACH="0.3", IB_RE="2000", IB_AOA="-4", IB_THICK="0.15",
               IB_NX="64", IB_LEVELS="3", IB_NPTS="120", IB_STEPS="0", IB_USER_INIT="0",
               IB_DUMP=os.path.join(work, "d"))
    out = subprocess.run([BINARY], cwd=work, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    d = pyoracle.read_dump(os.path.join(work, "d_000000.bin"))
    s = d["scalars"]
    assert abs(s[8] - 0.3) < 1e-15 and abs(s[9] - 2000.0) < 1e-9  # Ma, Re
    a = -4.0 / 180.0 * math.pi
    assert d["initvar"][1] == math.cos(a) and d["initvar"][2] == math.sin(a)
    # the 15 % profile is thicker: more cells inside the body than the 12 % one
    env["IB_THICK"] = "0.12"
    work2 = tempfile.mkdtemp(prefix="case_env_")
    env["IB_DUMP"] = os.path.join(work2, "d")
    assert subprocess.run([BINARY], cwd=work2, env=env, capture_output=True,
                          timeout=300).returncode == 0
    d2 = pyoracle.read_dump(os.path.join(work2, "d_000000.bin"))
    assert np.sum(d["signdis"] < 0) > np.sum(d2["signdis"] < 0)


def test_batched_airfoil_cases_span_the_stated_ranges():
    import bench
    c = bench.config4_cases()
    assert len(c) == 64 and c == bench.config4_cases()  # seeded
    mach = [float(e["IB_MACH"]) for e in c]
    aoa = [float(e["IB_AOA"]) for e in c]
    re = [float(e["IB_RE"]) for e in c]
    lev = {int(e["IB_LEVELS"]) for e in c}
    assert 0.1 <= min(mach) and max(mach) <= 0.8
    assert -5.0 <= min(aoa) and max(aoa) <= 10.0
    assert 2e3 <= min(re) and max(re) <= 2e4
    assert lev == {3, 4, 5, 6}  # the base grid and 2..5 AMR levels
    assert {e["IB_THICK"] for e in c[::2]} == {"0.12"} and {e["IB_THICK"] for e in c[1::2]} == {"0.15"}
    est = [int(e["IB_NX"]) ** 2 * bench.CONFIG4_LEAF_FACTOR[int(e["IB_LEVELS"])] for e in c]
    assert 4e4 <= min(est) and max(est) <= 9e5
