"""CPU checks of the refinement-indicator oracle (no GPU): the plain
criterion restatement against the tags the reference itself produced, the
oracle MLP's gradient against finite differences, and the package's rule
description against the oracle's."""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN_DIR, ORACLE_DIR

sys.path.insert(0, ORACLE_DIR)
import indicator_oracle as io  # noqa: E402

TAG_FIXTURES = [("naca_minmod_s4_n64_l3", 3), ("naca_tags_n64_l4", 4)]


def load_tags(name):
    with np.load(os.path.join(GOLDEN_DIR, name + ".npz")) as z:
        return z["tags"], z["dh"].reshape(-1, 3)[:, 0]


@pytest.mark.parametrize("name,nlev", TAG_FIXTURES)
def test_plain_criterion_oracle_matches_reference_tags(name, nlev):
    t, dh = load_tags(name)
    rule = io.naca_rule(nlev, dh)
    got = io.tag_plain(rule, t[:, 0].astype(int), t[:, 3], t[:, 4], t[:, 5])
    ref = io.tags_from_rftag(t[:, 6], t[:, 7])
    assert np.array_equal(got, ref), f"{np.sum(got != ref)} of {len(ref)} boxes differ"
    # the fixture exercises every branch: rectangles, bands, refine and coarsen
    assert np.any(ref & io.TAG_REFINE) and np.any(ref & io.TAG_COARSEN)
    assert np.any((t[:, 0] < nlev - 2) & ((ref & io.TAG_REFINE) != 0))
    assert np.any((t[:, 0] >= nlev - 2) & ((ref & io.TAG_REFINE) != 0))


def test_package_rule_matches_oracle_rule(pkg):
    for name, nlev in TAG_FIXTURES:
        _, dh = load_tags(name)
        a = pkg.workloads.naca_tag_rule(nlev, dh)
        b = io.naca_rule(nlev, dh)
        assert set(a) == set(b)
        for k in a:
            assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


def test_bf16_rounding_ties_to_even():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e-39])
    got = io.bf16_round(vals)
    assert got[0] == 1.0
    assert got[1] == 1.0                     # tie -> even
    assert got[2] == 1.0 + 4 * 2 ** -8       # tie -> even (up)
    assert got[3] == 1.0
    assert got[4] == -2.5
    assert io.bits_to_f64(io.bf16_bits(np.array([1.0])))[0] == 1.0


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    P = io.init_params(1).astype(np.float64)
    P[io.P_B1:io.P_W2] = rng.normal(0, 0.1, io.N_HID)
    X = rng.normal(0, 1, (40, io.N_IN))
    y = rng.integers(0, 3, 40)
    y[5] = 7  # outside 0..2: contributes nothing
    cw = np.array([1.0, 2.5, 0.5])
    loss, g, _ = io.mlp_loss_grad(P, y, cw, X=X, rounding=False)
    idx = np.concatenate([rng.choice(np.arange(io.P_W1, io.P_B1), 6), np.arange(io.P_B1, io.P_B1 + 3),
                          rng.choice(np.arange(io.P_W2, io.P_B2), 6), np.arange(io.P_B2, io.P_B2 + 3),
                          rng.choice(np.arange(io.P_W3, io.P_B3), 6), np.arange(io.P_B3, io.P_COUNT)])
    h = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        lp = io.mlp_loss_grad(Pp, y, cw, X=X, rounding=False)[0]
        lm = io.mlp_loss_grad(Pm, y, cw, X=X, rounding=False)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])
    assert loss > 0


def test_oracle_adam_step():
    P = np.ones(4)
    g = np.array([1.0, -1.0, 0.0, 2.0])
    P1, m, v = io.adam(P, g, np.zeros(4), np.zeros(4), 1, 0.1)
    # first bias-corrected step moves each weight by lr * sign(g)
    assert np.allclose(P1, [0.9, 1.1, 1.0, 0.9], atol=1e-6)
