"""Host logic of the serving loop (admission under the HBM budget, arrival
order, failures), with a stand-in fit that needs no GPU."""
import threading
import time

import numpy as np
import pytest

from ccd_b200 import serve, synthetic
from ccd_b200.data import MODEL_LOGISTIC


def _stub(duration=0.02, fail_on=()):
    lock = threading.Lock()
    live = {"now": 0, "peak": 0}

    def fit(slot, req, local):
        with lock:
            live["now"] += 1
            live["peak"] = max(live["peak"], live["now"])
        time.sleep(duration)
        with lock:
            live["now"] -= 1
        if req.rid in fail_on:
            raise RuntimeError("planted failure")
        return np.full(3, float(req.rid)), 0, 1, -1.0
    return fit, live


def _req(i, nbytes):
    d = synthetic.small(MODEL_LOGISTIC, seed=i, K=50, P=3)
    return serve.Request(i, d, bytes=nbytes)


def test_budget_bounds_concurrency_and_order_is_kept():
    fit, live = _stub()
    srv = serve.Server(hbm_budget=300, slots=8, fit_fn=fit)
    try:
        for i in range(12):
            srv.submit(_req(i, 100))  # three fit in the budget at a time
        done = srv.drain(12, timeout=30)
    finally:
        srv.close()
    assert len(done) == 12 and all(c.error is None for c in done)
    assert srv.peak_reserved <= 300 and live["peak"] <= 3 and srv.peak_running <= 3
    starts = [c.start for c in sorted(done, key=lambda c: c.rid)]
    assert starts == sorted(starts)  # admitted in arrival order
    assert all(np.array_equal(c.beta, np.full(3, float(c.rid))) for c in done)


def test_slots_bound_concurrency():
    fit, live = _stub()
    srv = serve.Server(hbm_budget=1 << 40, slots=2, fit_fn=fit)
    try:
        for i in range(6):
            srv.submit(_req(i, 10))
        srv.drain(6, timeout=30)
    finally:
        srv.close()
    assert live["peak"] <= 2


def test_failed_fit_is_reported_and_serving_continues():
    fit, _ = _stub(fail_on={1})
    srv = serve.Server(hbm_budget=1 << 40, slots=2, fit_fn=fit)
    try:
        for i in range(4):
            srv.submit(_req(i, 10))
        done = {c.rid: c for c in srv.drain(4, timeout=30)}
    finally:
        srv.close()
    assert "planted failure" in done[1].error
    assert all(done[i].error is None for i in (0, 2, 3))


def test_request_above_budget_is_refused():
    fit, _ = _stub()
    srv = serve.Server(hbm_budget=100, slots=1, fit_fn=fit)
    try:
        with pytest.raises(ValueError):
            srv.submit(_req(0, 101))
    finally:
        srv.close()


def test_latency_summary_and_stream_shape():
    stream = synthetic.serving_stream(12, seed=4, K_range=(1e3, 2e3), J_range=(20, 50))
    arrivals = [t for t, _ in stream]
    assert arrivals == sorted(arrivals)
    fit, _ = _stub(0.001)
    srv = serve.Server(hbm_budget=1 << 40, slots=3, fit_fn=fit)
    try:
        done = serve.replay(srv, stream, time_scale=0.01)
    finally:
        srv.close()
    s = serve.latency_summary(done)
    assert s["requests"] == 12 and s["failed"] == 0 and s["p99_s"] >= s["p50_s"] > 0


def test_fast_lane_takes_small_requests_ahead_of_large_ones():
    """One general slot busy with a queue of large requests; the fast slot
    serves the small requests that arrived after them, in their own arrival
    order, and never takes a large one."""
    taken = []
    lock = threading.Lock()

    def fit(slot, req, local):
        with lock:
            taken.append((slot, req.rid))
        time.sleep(0.15 if req.data.nnz > 400 else 0.005)
        return np.zeros(3), 0, 1, -1.0

    big = [serve.Request(i, synthetic.small(MODEL_LOGISTIC, seed=i, K=2000, P=10, density=0.1), bytes=1)
           for i in range(3)]
    small = [serve.Request(10 + i, synthetic.small(MODEL_LOGISTIC, seed=10 + i, K=50, P=3), bytes=1)
             for i in range(4)]
    assert all(r.data.nnz > 400 for r in big) and all(r.data.nnz <= 400 for r in small)
    srv = serve.Server(hbm_budget=1e9, slots=1, fast_slots=1, fast_entries=400, fit_fn=fit)
    try:
        for r in big + small:
            srv.submit(r)
        done = srv.drain(7, timeout=30)
    finally:
        srv.close()
    by_rid = {c.rid: c for c in done}
    # every small request finished before the last large one
    assert max(by_rid[r.rid].end for r in small) < max(by_rid[r.rid].end for r in big)
    # the fast slot (slot 1) took only small requests, in arrival order
    fast = [rid for s, rid in taken if s == 1]
    assert fast and all(rid >= 10 for rid in fast) and fast == sorted(fast)
    # the general slot kept arrival order over what it took
    general = [rid for s, rid in taken if s == 0]
    assert general == sorted(general)


def test_slot_cta_limits():
    """Fast slots take fast_ctas CTAs; general slots share the SMs the fast
    slots leave, capped by slot_ctas when it is set; the slots' CTAs together
    never exceed the SM count."""
    fit, _ = _stub()
    cases = [(dict(slots=8, fast_slots=4), 148, 18, 1),
             (dict(slots=8, fast_slots=4, fast_ctas=4), 148, 16, 4),
             (dict(slots=8, fast_slots=4, slot_ctas=8), 148, 8, 1),
             (dict(slots=3, fast_slots=0), 148, 49, None),
             (dict(slots=200, fast_slots=2), 148, 1, 1)]
    for kw, n_sm, general, fast in cases:
        srv = serve.Server(hbm_budget=1e9, fit_fn=fit, **kw)
        try:
            limits = [srv.slot_max_ctas(s, n_sm) for s in range(kw["slots"] + kw["fast_slots"])]
        finally:
            srv.close()
        assert limits[:kw["slots"]] == [general] * kw["slots"]
        assert limits[kw["slots"]:] == [fast] * kw["fast_slots"]
        if general * kw["slots"] >= kw["slots"] and kw["slots"] <= n_sm:
            assert sum(limits) <= n_sm


def test_request_records_timeline():
    """Per-request records of a replay: model, size, slot, and wait / service
    times consistent with the completion times, offsets from the first arrival."""
    fit, _ = _stub(duration=0.01)
    stream = [(0.0, synthetic.small(MODEL_LOGISTIC, seed=i, K=50, P=3)) for i in range(5)]
    srv = serve.Server(hbm_budget=1e9, slots=2, fit_fn=fit)
    try:
        done = serve.replay(srv, stream)
    finally:
        srv.close()
    recs = serve.request_records(stream, done)
    assert [r["rid"] for r in recs] == list(range(5))
    for r, c in zip(recs, sorted(done, key=lambda c: c.rid)):
        assert r["model"] == MODEL_LOGISTIC and r["K"] == 50 and r["J"] == stream[r["rid"]][1].J
        assert r["slot"] in (0, 1) and r["error"] is None
        assert r["wait_s"] >= 0 and r["service_s"] >= 0.01
        assert abs(r["end_s"] - r["start_s"] - r["service_s"]) < 1e-9
        assert abs(r["start_s"] - r["arrival_s"] - r["wait_s"]) < 1e-9
    assert min(r["arrival_s"] for r in recs) == 0.0
    assert serve.request_records(stream, []) == []
