"""The layout server's scheduler on the host, with plain functions as the work: every request completes with its
own result, requests overlap up to the slot count, the memory budget is never exceeded, a request that waits for
memory is not overtaken by later ones, and a failing request fails alone."""
import threading
import time

import pytest

from magnet_b200.serve import Server, latency_summary


def sleeper(active, peak, lock):
    def work(kind, payload, slot):
        with lock:
            active[0] += 1
            peak[0] = max(peak[0], active[0])
        time.sleep(payload[1])
        with lock:
            active[0] -= 1
        if kind == "fail":
            raise RuntimeError("planted failure")
        return (payload[0], slot)
    return work


def test_results_overlap_and_budget():
    active, peak, lock = [0], [0], threading.Lock()
    srv = Server(sleeper(active, peak, lock), slots=3, budget_bytes=100)
    futs = [srv.submit("t", (i, 0.02), nbytes=30, points=10) for i in range(12)]
    res = [f.result(timeout=30) for f in futs]
    srv.close()
    assert [r[0] for r in res] == list(range(12))
    assert {r[1] for r in res} <= {0, 1, 2}
    assert peak[0] == 3                       # three slots, 3 x 30 bytes fit the budget of 100
    assert srv.peak_reserved <= 100
    s = latency_summary(srv.done, "t")
    assert s["requests"] == 12 and s["p99_ms"] >= s["p50_ms"] > 0 and s["points_per_s"] > 0


def test_budget_limits_concurrency():
    active, peak, lock = [0], [0], threading.Lock()
    srv = Server(sleeper(active, peak, lock), slots=4, budget_bytes=100)
    futs = [srv.submit("t", (i, 0.02), nbytes=60) for i in range(6)]
    for f in futs:
        f.result(timeout=30)
    srv.close()
    assert peak[0] == 1 and srv.peak_reserved == 60   # two requests of 60 never fit together


def test_waiting_request_is_not_overtaken():
    active, peak, lock = [0], [0], threading.Lock()
    srv = Server(sleeper(active, peak, lock), slots=3, budget_bytes=100)
    first = srv.submit("t", ("a", 0.2), nbytes=50)     # holds half the budget for a while
    time.sleep(0.05)
    big = srv.submit("t", ("big", 0.01), nbytes=100)   # must wait for `first`
    time.sleep(0.02)
    small = srv.submit("t", ("small", 0.01), nbytes=10)  # would fit now, but is behind `big`
    for f in (first, big, small):
        f.result(timeout=30)
    srv.close()
    t = {r.payload[0]: r.t_start for r in srv.done}
    assert t["big"] <= t["small"]


def test_failure_is_isolated_and_oversize_is_refused():
    active, peak, lock = [0], [0], threading.Lock()
    srv = Server(sleeper(active, peak, lock), slots=2, budget_bytes=100)
    bad = srv.submit("fail", (0, 0.0), nbytes=10)
    good = srv.submit("t", (1, 0.0), nbytes=10)
    with pytest.raises(RuntimeError, match="planted failure"):
        bad.result(timeout=30)
    assert good.result(timeout=30)[0] == 1
    with pytest.raises(ValueError, match="more than the server's budget"):
        srv.submit("t", (2, 0.0), nbytes=101)
    srv.close()


def test_slot_that_fails_to_start_leaves_the_work_to_the_others():
    """a worker whose start-up raises (e.g. its device cannot be set) takes no requests while another slot
    works; when every slot fails, the requests fail instead of waiting forever"""
    def init_one_bad(slot):
        if slot == 0:
            raise RuntimeError("no device for slot 0")

    srv = Server(lambda kind, payload, slot: (payload, slot), slots=2, budget_bytes=100, init=init_one_bad)
    futs = [srv.submit("t", i, nbytes=10) for i in range(20)]
    assert [f.result(timeout=30) for f in futs] == [(i, 1) for i in range(20)]
    srv.close()

    def init_all_bad(slot):
        raise RuntimeError("no device")

    srv = Server(lambda kind, payload, slot: payload, slots=3, budget_bytes=100, init=init_all_bad)
    futs = [srv.submit("t", i, nbytes=10) for i in range(5)]
    for f in futs:
        with pytest.raises(RuntimeError, match="failed to start"):
            f.result(timeout=30)
    srv.close()
