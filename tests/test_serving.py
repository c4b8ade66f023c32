"""Host logic of the serving loop: request padding and the FIFO queue."""
import numpy as np
import pytest

from pastix_b200.serving import bucket, buckets, fifo_latencies


def test_buckets_cover_every_request_size():
    assert buckets(256) == [1, 2, 4, 8] + list(range(16, 257, 16))
    for k in range(1, 257):
        b = bucket(k)
        assert b >= k and b in buckets(256)
        assert b - k < max(k, 16)
    with pytest.raises(ValueError):
        bucket(0)


def test_fifo_latencies():
    lat = fifo_latencies([0.0, 1.0, 1.5, 10.0], [2.0, 1.0, 1.0, 1.0])
    assert np.allclose(lat, [2.0, 2.0, 2.5, 1.0])
    # idle server: latency = service time
    assert np.allclose(fifo_latencies([0, 5, 10], [1, 2, 3]), [1, 2, 3])


from pastix_b200.serving import ContinuousBatcher


def _fake_backend(calls):
    def backend(b):
        calls.append(b.shape[0])
        k = b.shape[0]
        # per column independent (like the solve and the refinement), service grows with columns
        return 2.0 * b + np.arange(b.shape[1])[None, :], {"berr": np.full(k, 1e-13), "ms": 10.0 + 0.5 * k}
    return backend


def _np_batcher(calls, max_cols):
    def split(x, ks):
        return [x[c0:c0 + k].copy() for c0, k in zip(np.cumsum([0] + ks[:-1]), ks)]
    return ContinuousBatcher(_fake_backend(calls), max_cols, lambda bs: np.concatenate(bs, axis=0), split)


def test_continuous_batching_admits_arrived_requests_into_shared_batches():
    rng = np.random.default_rng(3)
    n = 7
    reqs = [(float(t), rng.standard_normal((int(k), n)))
            for t, k in zip(np.cumsum(rng.exponential(0.004, 40)), rng.integers(1, 40, 40))]
    calls = []
    out, batches = _np_batcher(calls, 64).run(reqs)
    served = sorted(i for b in batches for i in b["requests"])
    assert served == list(range(len(reqs)))                      # every request once
    assert all(b["cols"] <= 64 for b in batches)                   # slots
    assert max(len(b["requests"]) for b in batches) > 1            # requests share batches
    t_prev = 0.0
    for bi, b in enumerate(batches):
        start = out[b["requests"][0]]["start"]
        assert start >= t_prev - 1e-12
        for i in b["requests"]:
            assert reqs[i][0] <= start + 1e-12                    # admitted after arriving
        t_prev = start + b["service"]
    for i, (t, b) in enumerate(reqs):
        o = out[i]
        # the same result as alone
        assert np.array_equal(o["x"], 2.0 * b + np.arange(n)[None, :])
        assert o["x"].shape == b.shape and o["berr"].shape == (b.shape[0],)
        assert np.isclose(o["latency"], o["done"] - t) and o["latency"] > 0


def test_continuous_batching_fifo_admission_and_capacity():
    n = 3
    # three requests arrive together; the second does not fit next to the first
    reqs = [(0.0, np.ones((30, n))), (0.0, np.ones((40, n))), (0.0, np.ones((20, n))), (1.0, np.ones((5, n)))]
    calls = []
    out, batches = _np_batcher(calls, 64).run(reqs)
    assert [b["requests"] for b in batches] == [[0], [1, 2], [3]]
    assert calls == [30, 60, 5]
    # the late request starts when it arrives, the queue being empty by then
    assert out[3]["start"] == 1.0
    with pytest.raises(ValueError):
        _np_batcher([], 16).run([(0.0, np.ones((17, n)))])


def test_continuous_batching_orders_refactorizations():
    """Requests before a refactorization are served with the old factor, requests
    after it with the new one, whatever the batching."""
    from pastix_b200.serving import Refactor
    state = {"version": 1.0}
    calls = []

    def backend(b):
        calls.append(("solve", b.shape[0]))
        return state["version"] * b, {"berr": np.zeros(b.shape[0]), "ms": 5.0}

    def refactor(values):
        calls.append(("refactor", float(values[0])))
        state["version"] = float(values[0])
        return {"ms": 20.0}

    def split(x, ks):
        return [x[c0:c0 + k].copy() for c0, k in zip(np.cumsum([0] + ks[:-1]), ks)]

    bat = ContinuousBatcher(backend, 64, lambda bs: np.concatenate(bs, axis=0), split, refactor=refactor)
    n = 4
    reqs = [(0.000, np.ones((3, n))), (0.001, np.ones((2, n))), (0.002, Refactor(np.array([2.0]))),
            (0.003, np.ones((4, n))), (0.004, np.ones((1, n))), (0.050, Refactor(np.array([3.0]))),
            (0.051, np.ones((2, n)))]
    out, batches = bat.run(reqs)
    assert np.all(out[0]["x"] == 1.0) and np.all(out[1]["x"] == 1.0)
    assert np.all(out[3]["x"] == 2.0) and np.all(out[4]["x"] == 2.0)
    assert np.all(out[6]["x"] == 3.0)
    assert out[2]["refactor"]["ms"] == 20.0 and out[2]["done"] <= out[3]["start"] + 1e-12
    # requests 3 and 4 arrived during the refactorization: served together after it
    assert [b["requests"] for b in batches][:4] == [[0], [1], [2], [3, 4]]
    with pytest.raises(ValueError):
        ContinuousBatcher(backend, 64, None, None).run([(0.0, Refactor(np.array([1.0])))])
