"""Admission of the serving loop (host logic, no GPU): one FIFO queue per
model under one memory budget; a request waiting for memory does not hold up
other models' requests until it has waited max_bypass_s, then nothing younger
goes ahead of it; cancelling removes a waiting request."""
import numpy as np

from tclb_b200.batch import CaseSpec
from tclb_b200.serve import Admission, Request


def _req(rid, model, fp, arrival):
    spec = CaseSpec(np.zeros((1, 1, 1), np.uint16), {}, {}, 10)
    r = Request(rid, model, spec, arrival)
    r.fp = fp
    return r


def _adm(budget=100, bypass=5.0):
    return Admission(budget, lambda r: r.fp, ("d2q9", "d3q19"), max_bypass_s=bypass)


def test_other_models_go_ahead_of_a_request_waiting_for_memory():
    a = _adm()
    big, waits, small = _req(0, "d3q19", 80, 0.0), _req(1, "d3q19", 50, 1.0), _req(2, "d2q9", 10, 2.0)
    for r in (big, waits, small):
        a.submit(r)
    assert a.admit(0.5) == [big]
    assert a.admit(2.5) == [small]  # the waiting d3q19 request does not block d2q9
    assert a.used == 90 and a.waiting() == 1
    a.release(big)
    assert a.admit(3.0) == [waits]
    assert a.used == 60


def test_a_request_that_waited_long_enough_reserves_the_memory():
    a = _adm(bypass=5.0)
    big, waits = _req(0, "d3q19", 80, 0.0), _req(1, "d3q19", 50, 1.0)
    late = _req(2, "d2q9", 10, 7.0)
    for r in (big, waits, late):
        a.submit(r)
    assert a.admit(1.0) == [big]  # waits starts waiting for memory at t = 1
    assert a.admit(7.0) == []  # it has waited 6 s >= 5 s: the younger d2q9 request stays queued
    a.release(big)
    assert a.admit(7.5) == [waits, late]  # oldest first once memory is free


def test_arrival_order_and_not_yet_arrived():
    a = _adm(budget=1000)
    rs = [_req(i, "d2q9" if i % 2 else "d3q19", 10, 0.5 * i) for i in range(6)]
    for r in rs:
        a.submit(r)
    assert [r.rid for r in a.admit(1.2)] == [0, 1, 2]
    assert [r.rid for r in a.admit(10.0)] == [3, 4, 5]


def test_cancel_a_waiting_request():
    a = _adm()
    big, waits, other = _req(0, "d3q19", 80, 0.0), _req(1, "d3q19", 50, 0.1), _req(2, "d3q19", 10, 0.2)
    for r in (big, waits, other):
        a.submit(r)
    assert a.admit(0.0) == [big]
    assert a.cancel(1) is waits
    assert a.cancel(1) is None
    assert a.admit(0.3) == [other]  # the queue moved on past the cancelled request
    assert a.waiting() == 0


def test_request_above_the_whole_budget_is_refused():
    import pytest

    from tclb_b200.batch import AdmissionRefused

    a = _adm(budget=100)
    with pytest.raises(AdmissionRefused):
        a.submit(_req(0, "d2q9", 101, 0.0))
