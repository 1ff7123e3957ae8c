"""Served request loop (continuous batching) on a GPU.

Requests arrive while earlier ones are on the device; each result must equal the result of the
same problem solved alone (2D: the batched engine with that problem alone; 3D: the complex64
plane engine), bit for bit, since every item is computed by the same kernel independently of
its neighbours. Admission keeps the device memory of the requests in flight within the budget.
"""

from __future__ import annotations

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _alone_2d(prob):
    from bwpm_b200.batch import Batch2D

    b = Batch2D()
    i = b.add_problem(prob)
    b.run()
    return b.result(i)


def _alone_3d(prob):
    from bwpm_b200 import _core

    s = _core.CudaSolver(*prob.core_args(), 0, precision=32)
    return s.run(prob.field, prob.iterations, [])


def _stream():
    from bwpm_b200 import workloads

    probs = workloads.batch2d(count=10, seed=21, sizes=(256, 384, 1024, 1536, 3000),
                              nz_range=(30, 90), iterations=2)
    probs.insert(3, workloads.microlens3d(n=48, nz=40, iterations=2))
    probs.insert(7, workloads.microlens3d(n=32, nz=24, iterations=1))
    return probs


def test_served_results_equal_alone_and_in_mix():
    from bwpm_b200.serve import Server

    probs = _stream()
    with Server(max_group_solves=3) as srv:
        tickets = []
        for k, p in enumerate(probs):
            tickets.append(srv.submit(p))
            time.sleep(0.002 * (k % 3))  # staggered arrivals: later requests meet running ones
        results = [srv.result(t) for t in tickets]
        st = srv.stats()
    assert st["completed"] == len(probs) and st["failed"] == 0
    assert st["groups"] >= 2
    assert st["max_concurrent"] >= 2
    for p, r in zip(probs, results):
        assert r["latency_ms"] >= r["queue_ms"] >= 0.0
        if p.nx == 1:
            a = _alone_2d(p)
            assert np.array_equal(r["transmitted"], a["transmitted"]), p.name
            assert np.array_equal(r["reflected"], a["reflected"]), p.name
            assert np.allclose(r["energy_residual"], a["energy_residual"], rtol=0, atol=0)
        else:
            a = _alone_3d(p)
            assert np.array_equal(r["transmitted"], a["transmitted"]), p.name
            assert np.array_equal(r["reflected"], a["reflected"]), p.name


def test_served_admission_keeps_the_budget():
    from bwpm_b200 import workloads
    from bwpm_b200.serve import Server

    probs = workloads.batch2d(count=8, seed=22, sizes=(1024, 2048), nz_range=(40, 60),
                              iterations=1)
    budget = 3 << 20  # a few requests at a time
    with Server(budget_bytes=budget) as srv:
        tickets = [srv.submit(p) for p in probs]
        results = [srv.result(t) for t in tickets]
        st = srv.stats()
    assert st["completed"] == len(probs)
    assert st["peak_bytes"] <= budget
    assert st["groups"] >= 2  # the budget split the stream into several launches
    for p, r in zip(probs, results):
        a = _alone_2d(p)
        assert np.array_equal(r["transmitted"], a["transmitted"])


def test_served_failed_request_does_not_stop_the_others():
    from bwpm_b200 import workloads
    from bwpm_b200.serve import Server

    good = workloads.batch2d(count=3, seed=23, sizes=(256,), nz_range=(20, 30), iterations=1)
    bad = workloads.batch2d(count=1, seed=24, sizes=(256,), nz_range=(20, 30), iterations=1)[0]
    bad.labels = bad.labels.copy()
    bad.labels[0, 0, 0] = 7  # no such material
    with Server() as srv:
        t0 = srv.submit(good[0])
        tb = srv.submit(bad)
        t1, t2 = srv.submit(good[1]), srv.submit(good[2])
        with pytest.raises(RuntimeError, match="labels must index"):
            srv.result(tb)
        for t, p in zip((t0, t1, t2), good):
            assert np.array_equal(srv.result(t)["transmitted"], _alone_2d(p)["transmitted"])
        st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 3


def test_borrowed_and_copied_submissions_give_the_same_results():
    """Borrowed labels (copied later by the server's preparation workers) and labels copied in
    the call give the same results, 2D and 3D, and the caller's own array may go away at once."""
    from bwpm_b200.serve import Server

    probs = _stream()[:6]
    with Server() as srv:
        copied = [srv.result(srv.submit(p, borrow=False)) for p in probs]
    with Server() as srv:
        tickets = []
        for p in probs:
            # a private copy that only the Server keeps alive after the call
            q = type(p)(**{**p.__dict__, "labels": np.array(p.labels, copy=True)})
            tickets.append(srv.submit(q))
            del q
        borrowed = [srv.result(t) for t in tickets]
    for p, a, b in zip(probs, copied, borrowed):
        assert np.array_equal(a["transmitted"], b["transmitted"]), p.name
        assert np.array_equal(a["reflected"], b["reflected"]), p.name
