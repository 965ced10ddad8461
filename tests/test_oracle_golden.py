"""The CPU oracle (C restatement) against the reference solver's own output.

The golden fixtures were produced by running the reference sources
(tests/golden/make_golden.py); the restatement must reproduce every dumped
step bit for bit, which pins it before the GPU path is tested against it.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402

GOLDEN = [("vortex_vanleer_s4_n32", 0), ("vortex_minmod_s3_n32", 1)]


@pytest.mark.parametrize("name,limiter", GOLDEN)
def test_oracle_reproduces_reference_bitwise(oracle, name, limiter):
    g = make_golden.load(name)
    nsnap = g["prim"].shape[0]
    for k in range(nsnap - 1):
        d0 = make_golden.snapshot(g, k)
        P = oracle.params_from_dump(d0, limiter, viscous=False)
        lv = oracle.OracleLevels(d0)
        rc, dt, cfl, res = oracle.step(P, lv, k, d0["scalars"][1])
        assert rc == 0
        d1 = make_golden.snapshot(g, k + 1)
        assert dt == d1["scalars"][1]
        got = lv.state_like_dump(d1)
        ref = g["prim"][k + 1]
        assert np.array_equal(got, ref), f"step {k}: max diff {np.abs(got - ref).max()}"


def test_oracle_flags_match_product_flags(oracle, pkg):
    """The oracle's and the product's reading of the reference box attributes
    agree (two independent restatements of the same branch structure)."""
    rng = np.random.default_rng(0)
    n = 2000
    kind = rng.integers(0, 4, n)
    solid = rng.integers(0, 2, n)
    infect = np.where(rng.random(n) < 0.3, rng.integers(0, 50, n), -1)
    signdis = rng.normal(size=n)
    for body in (False, True):
        a = oracle.cell_flags(kind, solid, infect, signdis, body)
        b = pkg.ibgpu.cell_flags_from_boxes(kind, solid, infect, signdis, body)
        assert np.array_equal(a, b & 0x3f)
