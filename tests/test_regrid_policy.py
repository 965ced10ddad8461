"""The learned indicator's deployment policy (indicator.Regridder) on CPU,
with the tagging calls replaced by fakes: the learned decision on ordinary
regrids, the plain criterion's tags on every judge_every-th regrid (the
first included) with the learned decision's mismatch recorded, and the
plain criterion on every regrid when judge_every is 1."""
import numpy as np

from conftest import load_pkg

pkg = load_pkg()
ib, ind = pkg.ibgpu, pkg.indicator

PLAIN = np.array([ib.TAG_REFINE, 0, ib.TAG_COARSEN, 0], np.uint8)
LEARNED = np.array([ib.TAG_REFINE, ib.TAG_REFINE, ib.TAG_COARSEN, 0], np.uint8)  # 1 of 4 differs


class FakeSolver:
    def __init__(self):
        self.plain_calls = 0

    def tag_plain(self, rule, level, xc, yc, signdis, ix=None, iy=None):
        self.plain_calls += 1
        return PLAIN.copy()


class FakeIndicator:
    def __init__(self):
        self.solver = FakeSolver()
        self.calls = 0

    def tags(self, rule, boxes):
        self.calls += 1
        return LEARNED.copy()


BOXES = dict(level=np.zeros(4, np.int32), ix=np.arange(4, dtype=np.int32),
             iy=np.zeros(4, np.int32), xc=np.zeros(4), yc=np.zeros(4), signdis=np.ones(4))


def test_plain_criterion_rejudges_every_nth_regrid():
    fi = FakeIndicator()
    rg = ind.Regridder(fi, rule={}, judge_every=10)
    used = [rg.tags(BOXES) for _ in range(25)]
    judged = [k for k, t in enumerate(used) if np.array_equal(t, PLAIN)]
    assert judged == [0, 10, 20]
    assert all(np.array_equal(used[k], LEARNED) for k in range(25) if k not in judged)
    assert fi.solver.plain_calls == 3 and fi.calls == 25  # the learned decision every time
    assert rg.mismatch == [(0, 0.25), (10, 0.25), (20, 0.25)]


def test_judge_every_one_is_the_plain_criterion():
    fi = FakeIndicator()
    rg = ind.Regridder(fi, rule={}, judge_every=1)
    assert all(np.array_equal(rg.tags(BOXES), PLAIN) for _ in range(5))
    assert len(rg.mismatch) == 5


def test_classes_and_tags_round_trip():
    cls = np.array([ind.CLASS_REFINE, ind.CLASS_COARSEN, ind.CLASS_KEEP], np.uint8)
    assert np.array_equal(ind.classes_from_tags(ind.tags_from_classes(cls)), cls)
    # refine wins over coarsen in the plain criterion's bits
    both = np.array([ib.TAG_REFINE | ib.TAG_COARSEN], np.uint8)
    assert ind.classes_from_tags(both)[0] == ind.CLASS_REFINE
