"""Host-side object lifetimes of the Python front end (no GPU): a batch runs
on its first case's stream and holds its cases' contexts, so closing a case
destroys every batch holding it first.  The C library is replaced by a fake
that records the calls."""
import pytest

PARAMS = dict(nstages=4, tp=[0.25, 1 / 3, 0.5, 1.0], initvar=[1.0, 0.5, 0.0, 0.0, 1 / 1.4, 1.0, 0.0],
              nlevels=1, dh=[[0.1, 0.1, 1.0]], march_step=[1], march_left=[0], step_num=[1.0],
              domain_nx=32, domain_ny=32, periodic_x=1, periodic_y=1)


class FakeLib:
    def __init__(self):
        self.calls = []
        self.next = 100

    def _handle(self, ref):
        self.next += 1
        ref._obj.value = self.next
        return self.next

    def ibgpu_create(self, case_ref, ctx_ref):
        self.calls.append(("create", self._handle(ctx_ref)))
        return 0

    def ibgpu_batch_create(self, arr, n, b_ref):
        self.calls.append(("batch_create", self._handle(b_ref), tuple(arr[i] for i in range(n))))
        return 0

    def ibgpu_destroy(self, ctx):
        self.calls.append(("destroy", ctx.value))

    def ibgpu_batch_destroy(self, b):
        self.calls.append(("batch_destroy", b.value))

    def ibgpu_last_error(self):
        return b""


@pytest.fixture
def fake(pkg, monkeypatch):
    f = FakeLib()
    monkeypatch.setattr(pkg.ibgpu, "_lib", f)
    return f


def test_closing_a_case_destroys_its_batches_first(pkg, fake):
    ib = pkg.ibgpu
    a, b = ib.FlowSolver(PARAMS), ib.FlowSolver(PARAMS)
    batch = ib.Batch([a, b])
    ha, hb = a._ctx.value, batch._b.value
    a.close()
    assert fake.calls[-2:] == [("batch_destroy", hb), ("destroy", ha)]
    assert not batch._b
    batch.close()  # already gone: no second destroy
    b.close()
    kinds = [c[0] for c in fake.calls]
    assert kinds.count("batch_destroy") == 1
    assert kinds.count("destroy") == 2


def test_closed_batch_is_forgotten_by_its_cases(pkg, fake):
    ib = pkg.ibgpu
    a = ib.FlowSolver(PARAMS)
    batch = ib.Batch([a])
    batch.close()
    del batch
    a.close()
    assert [c[0] for c in fake.calls] == ["create", "batch_create", "batch_destroy", "destroy"]
