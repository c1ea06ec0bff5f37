"""Continuous-batching server: requests that arrive while others run are
admitted as memory frees up, and each result is the same alone and in the mix
(velocity relative L2 <= 1e-6 FP32: identical node arithmetic; Globals within
1e-9 relative, FP64 sums in a different order)."""
import numpy as np
import pytest

from tclb_b200 import cases
from tclb_b200.batch import CaseSpec, case_bytes
from tclb_b200.serve import Request, Server

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def small_requests():
    reqs = []
    d2, _ = cases.batch_cases_d2q9(6, seed=3, w_min=64, w_max=256)
    for i, c in enumerate(d2):
        fl = cases.disc_channel_flags(c["W"], c["H"], c["r"], c["cx"], c["cy"])
        spec = CaseSpec(fl, {"Viscosity": c["nu"]}, {0: {"VelocityX": c["ux"]}, 1: {"VelocityX": c["ux"]}},
                        40 + 17 * i)
        reqs.append(Request(i, "d2q9", spec, arrival=0.01 * i, want_quantity="U"))
    for j, n in enumerate((32, 64)):
        fl = cases.porous_channel_d3q19(n, n, n, p=0.1, band=2, seed=j)
        spec = CaseSpec(fl, {"nu": 0.02, "ForceX": 1e-5}, {}, 50 + 30 * j)
        reqs.append(Request(6 + j, "d3q19", spec, arrival=0.005 + 0.02 * j, want_quantity="U"))
    return reqs


def test_results_same_alone_and_in_the_mix():
    launch = {"d2q9": (64, 4, 16), "d3q19": (32, 8, 8)}
    reqs = small_requests()
    # a budget that holds only part of the mix: later requests wait for memory
    fps = [case_bytes(r.model, *r.spec.shape[::-1]) for r in reqs]
    budget = max(fps) + sorted(fps)[-2]
    srv = Server(("d2q9", "d3q19"), "fp32", "same", budget_bytes=budget, launch=launch)
    rep = srv.run(reqs)
    srv.close()
    assert rep["requests"] == len(reqs) and rep["pending"] == 0
    assert all(r.finished >= r.admitted >= 0 for r in reqs)
    assert any(r.admitted - r.arrival > 0.0 for r in reqs)  # some request waited for memory
    for r in (reqs[2], reqs[7]):
        alone = Server((r.model,), "fp32", "same", budget_bytes=1 << 30, launch=launch)
        r2 = Request(r.rid, r.model, r.spec, 0.0, want_quantity="U")
        alone.run([r2])
        alone.close()
        assert rel_l2(r.quantity, r2.quantity) <= 1e-6
        assert np.allclose(r.globals, r2.globals, rtol=1e-9, atol=1e-15)


def test_cancel_waiting_pending_and_running_requests():
    """A request cancelled while it waits for memory never runs; one cancelled
    while it runs leaves at its batch's next boundary; the others finish with
    the same results as without the cancellations, and all memory is returned."""
    launch = {"d2q9": (64, 4, 16), "d3q19": (32, 8, 8)}
    reqs = small_requests()
    r1 = reqs[1]  # long enough to be running when it is cancelled at t = 0.06 s (it arrives at 0.01 s)
    r1.spec = CaseSpec(r1.spec.flags, r1.spec.settings, r1.spec.zone_settings, 200000)
    fps = [case_bytes(r.model, *r.spec.shape[::-1]) for r in reqs]
    budget = max(fps) + sorted(fps)[-2]
    srv = Server(("d2q9", "d3q19"), "fp32", "same", budget_bytes=budget, launch=launch)
    # request 7 is cancelled before it arrives (still queued), request 1 while it runs
    rep = srv.run(reqs, cancels=[(0.0, 7), (0.06, 1)])
    srv.close()
    by_id = {r.rid: r for r in reqs}
    assert rep["pending"] == 0 and srv.used == 0
    assert rep["requests"] + rep["cancelled"] == len(reqs)
    assert by_id[7].cancelled and by_id[7].globals is None
    assert by_id[1].cancelled and by_id[1].globals is None
    for r in reqs:
        if not r.cancelled:
            assert r.globals is not None and r.quantity is not None
    # an uncancelled request gives the same result as when served alone
    r = by_id[2]
    alone = Server((r.model,), "fp32", "same", budget_bytes=1 << 30, launch=launch)
    r2 = Request(r.rid, r.model, r.spec, 0.0, want_quantity="U")
    alone.run([r2])
    alone.close()
    assert rel_l2(r.quantity, r2.quantity) <= 1e-6


def test_large_requests_as_their_own_lattice():
    """With solo_nodes, requests of at least that many nodes run as lattices of their
    own (in chunks on their own streams) while the rest are batched: every result is
    the one the batched path gives, and a large request cancelled while it runs
    leaves with its memory returned."""
    launch = {"d2q9": (64, 4, 16), "d3q19": (32, 8, 8)}
    reqs = small_requests()  # d3q19 boxes of 32^3 and 64^3 nodes; 64^3 runs as its own lattice
    budget = 4 << 30
    solo = Server(("d2q9", "d3q19"), "fp32", "same", budget_bytes=budget, launch=launch, solo_nodes=64 ** 3,
                  solo_iters=7)
    rep = solo.run(reqs)
    solo.close()
    assert rep["requests"] == len(reqs) and rep["pending"] == 0 and solo.used == 0
    ref = [Request(r.rid, r.model, r.spec, r.arrival, want_quantity="U") for r in small_requests()]
    batched = Server(("d2q9", "d3q19"), "fp32", "same", budget_bytes=budget, launch=launch)
    batched.run(ref)
    batched.close()
    for r, q in zip(reqs, ref):
        assert rel_l2(r.quantity, q.quantity) <= 1e-6, r.rid
        assert np.allclose(r.globals, q.globals, rtol=1e-9, atol=1e-15), r.rid
    # cancel the large request while it runs
    reqs = small_requests()
    big = reqs[7]
    big.spec = CaseSpec(big.spec.flags, big.spec.settings, big.spec.zone_settings, 200000)
    srv = Server(("d2q9", "d3q19"), "fp32", "same", budget_bytes=budget, launch=launch, solo_nodes=64 ** 3)
    rep = srv.run(reqs, cancels=[(0.2, 7)])
    srv.close()
    assert big.cancelled and big.globals is None
    assert rep["requests"] == len(reqs) - 1 and rep["pending"] == 0 and srv.used == 0
