"""Host logic of requests served as lattices of their own (Server._step_solo), on the CPU.

A fake lattice records the iterations it is asked for and a fake CUDA event
reports its chunk done, so the bookkeeping is tested without a GPU: the
iterations of a request are run in chunks of solo_iters, the last one alone
with ITER_LASTGLOB (its Globals), the lattice is closed and the memory
returned when it finishes, and a cancelled request leaves after its chunk in
flight without Globals.
"""
import numpy as np
import pytest

from tclb_b200 import models as M
from tclb_b200.batch import CaseSpec
from tclb_b200.serve import Admission, Request, Server, _Solo


class FakeLattice:
    def __init__(self):
        self.calls, self.closed = [], False

    def Iterate(self, n, iter_type=M.ITER_NORM, stream=0):
        assert not self.closed
        self.calls.append((n, iter_type))

    @property
    def globals(self):
        return np.array([1.0, 2.0])

    def GetQuantity(self, name):
        return np.zeros(4)

    def close(self):
        self.closed = True


class FakeStream:
    cuda_stream = 0


class FakeEvent:
    ready = True

    def record(self, stream):
        pass

    def query(self):
        return FakeEvent.ready


@pytest.fixture
def server(monkeypatch):
    import torch

    monkeypatch.setattr(torch.cuda, "Event", FakeEvent)
    srv = Server.__new__(Server)  # the host state only: no batches, no GPU
    srv.adm = Admission(1 << 30, lambda r: 1000, ("d3q19",))
    srv.solo, srv.solo_iters, srv.done, srv.cancelled = {}, 4, [], []
    import time
    srv.t0 = time.perf_counter()
    return srv


def _request(niter, quantity=None):
    spec = CaseSpec(np.zeros((2, 2, 2), np.uint16), {}, {}, niter)
    return Request(0, "d3q19", spec, 0.0, want_quantity=quantity)


def _run(srv, rid, limit=100):
    for _ in range(limit):
        if rid not in srv.solo:
            return
        srv._step_solo(srv.solo[rid])
    raise AssertionError("did not finish")


@pytest.mark.parametrize("niter", [0, 1, 2, 4, 5, 9, 10, 64])
def test_chunks_and_last_iteration_with_globals(server, niter):
    r = _request(niter, quantity="U")
    server.adm.used = 1000  # as admitted
    lat = FakeLattice()
    server.solo[r.rid] = _Solo(r, lat, FakeStream(), niter)
    _run(server, r.rid)
    assert sum(n for n, _ in lat.calls) == niter
    assert all(n <= server.solo_iters for n, _ in lat.calls)
    lastglob = [t & M.ITER_LASTGLOB for _, t in lat.calls]
    if niter:
        assert lat.calls[-1] == (1, M.ITER_NORM | M.ITER_LASTGLOB) and sum(1 for g in lastglob if g) == 1
    assert lat.closed and server.done == [r] and r.globals is not None and r.quantity is not None
    assert server.adm.used == 0 and r.finished >= 0


def test_chunk_in_flight_is_waited_for(server):
    r = _request(20)
    lat = FakeLattice()
    server.adm.used = 1000
    server.solo[r.rid] = _Solo(r, lat, FakeStream(), 20)
    FakeEvent.ready = False
    try:
        assert server._step_solo(server.solo[r.rid])  # enqueues the first chunk
        for _ in range(5):
            assert not server._step_solo(server.solo[r.rid])  # still in flight: nothing happens
        assert lat.calls == [(4, M.ITER_NORM)]
    finally:
        FakeEvent.ready = True
    _run(server, r.rid)
    assert sum(n for n, _ in lat.calls) == 20


def test_cancel_leaves_after_the_chunk_in_flight(server):
    r = _request(1000)
    lat = FakeLattice()
    server.adm.used = 1000
    server.solo[r.rid] = _Solo(r, lat, FakeStream(), 1000)
    server._step_solo(server.solo[r.rid])
    server.solo[r.rid].cancel = True
    _run(server, r.rid)
    assert r.cancelled and r.globals is None and lat.closed
    assert server.cancelled == [r] and server.done == [] and server.adm.used == 0
    assert all(t == M.ITER_NORM for _, t in lat.calls)


def test_reserve_above_the_budget_is_refused():
    """The pools set aside at start-up must fit the budget; checked before any batch is made."""
    with pytest.raises(ValueError):
        Server(("d2q9", "d3q19"), budget_bytes=1 << 20, reserve={"d2q9": 1 << 19, "d3q19": 1 << 20})
