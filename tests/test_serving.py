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
