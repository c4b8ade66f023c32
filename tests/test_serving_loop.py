"""Host logic of the real-time serving loop (ServingLoop), on CPU with a fake
backend that sleeps for its service times: requests submitted while batches run
are admitted into idle lanes in arrival order, batches on different lanes overlap,
requests before a refactorization are served by the old factor and those after it
by the new one, a refactorization goes into the standby factor at once (while the
old one still serves) when there is one and in place after the old epoch drains
when there is not, and a backend failure reaches the caller."""
import threading
import time

import numpy as np
import pytest

from pastix_b200.serving import Refactor, ServingLoop, poisson_offsets, replay


class FakeBackend:
    def __init__(self, lanes=2, max_cols=8, slots=2, service=0.03, refactor_s=0.08):
        self.lanes, self.max_cols, self.slots = lanes, max_cols, slots
        self.tag = {0: "A"}
        self.service, self.refactor_s = service, refactor_s
        self.lock = threading.Lock()
        self.active = 0
        self.max_active = 0
        self.log = []
        self.fail = False

    def standby_ok(self, slot):
        return slot < self.slots

    def refactor(self, slot, values):
        t0 = time.perf_counter()
        time.sleep(self.refactor_s)
        with self.lock:
            self.tag[slot] = values
            self.log.append(("refactor", slot, values, t0, time.perf_counter()))
        return dict(ms=(time.perf_counter() - t0) * 1e3)

    def solve(self, slot, lane, blocks):
        if self.fail:
            raise RuntimeError("device failure")
        with self.lock:
            self.active += 1
            self.max_active = max(self.max_active, self.active)
            tag = self.tag[slot]
        t0 = time.perf_counter()
        time.sleep(self.service)
        with self.lock:
            self.active -= 1
            self.log.append(("solve", slot, lane, t0, time.perf_counter()))
        return [(tag, b) for b in blocks], [np.zeros(b.shape[0]) for b in blocks], dict(iters=1)


def req(k, i):
    return np.full((k, 3), float(i))


def test_lanes_overlap_and_arrival_order():
    be = FakeBackend()
    loop = ServingLoop(be)
    ks = [3, 4, 2, 5, 1, 6, 2, 3]
    for i, k in enumerate(ks):
        loop.submit(req(k, i))
    res = loop.drain(30)
    loop.close()
    assert be.max_active == 2
    done = []
    for b in loop.batches:
        assert b["cols"] <= be.max_cols
        assert b["requests"] == sorted(b["requests"])
        done += b["requests"]
    assert done == list(range(len(ks)))  # admitted in arrival order
    for i, k in enumerate(ks):
        tag, blk = res[i]["x"]
        assert tag == "A" and blk.shape == (k, 3) and blk[0, 0] == i
        assert res[i]["latency"] >= be.service


@pytest.mark.parametrize("slots", [2, 1])
def test_refactor_epochs_standby_and_in_place(slots):
    be = FakeBackend(slots=slots, service=0.05, refactor_s=0.08)
    loop = ServingLoop(be)
    items = [req(2, 0), req(3, 1), Refactor("B"), req(2, 3), req(1, 4), Refactor("C"), req(2, 6)]
    for it in items:
        loop.submit(it)
    res = loop.drain(30)
    loop.close()
    want = {0: "A", 1: "A", 3: "B", 4: "B", 6: "C"}
    for i, tag in want.items():
        assert res[i]["x"][0] == tag, (i, res[i]["x"][0])
    r1, r2 = res[2], res[5]
    assert r1["refactor"] and r2["refactor"]
    first_solve_end = max(res[0]["done"], res[1]["done"])
    if slots == 2:
        # the standby factor is refactored while the old one still serves
        assert r1["slot"] == 1 and r1["standby"]
        assert r1["start"] < first_solve_end
        assert r2["slot"] == 0
    else:
        assert r1["slot"] == 0 and not r1["standby"]
        assert r1["start"] >= first_solve_end - 1e-6
    # requests of a later epoch finish after their factor was ready
    assert min(res[3]["done"], res[4]["done"]) >= r1["done"]
    assert res[6]["done"] >= r2["done"]


def test_realtime_arrivals_from_a_producer_thread():
    be = FakeBackend(service=0.01)
    loop = ServingLoop(be)
    offs = poisson_offsets(20, 200.0, seed=3)
    trace = [(o, req(1 + (i % 4), i)) for i, o in enumerate(offs)]
    th = replay(loop, trace)
    th.join()
    res = loop.drain(30)
    loop.close()
    lat = np.array([res[i]["latency"] for i in range(20)])
    arr = np.array([res[i]["arrival"] for i in range(20)])
    assert np.all(np.diff(arr) >= 0)                      # submitted in trace order
    assert arr[-1] == pytest.approx(offs[-1], abs=0.25)     # at wall-clock offsets
    assert np.all(lat >= be.service)
    assert len(loop.batches) < 20                           # some requests shared a batch


def test_backend_failure_reaches_drain():
    be = FakeBackend()
    be.fail = True
    loop = ServingLoop(be)
    loop.submit(req(2, 0))
    with pytest.raises(RuntimeError, match="device failure"):
        loop.drain(10)
    loop.close()


def test_oversized_request_refused():
    loop = ServingLoop(FakeBackend(max_cols=4))
    with pytest.raises(ValueError):
        loop.submit(req(5, 0))
    loop.close()
