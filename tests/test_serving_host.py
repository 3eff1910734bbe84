"""Host logic of batching and serving that needs no GPU: the arena's segment allocator and requests."""

from __future__ import annotations

import numpy as np
import pytest

from offline_particles_b200.batching import SegmentAllocator
from offline_particles_b200.serving import ReleaseRequest


def test_segment_allocator_first_fit_and_coalescing():
    a = SegmentAllocator(100)
    s1 = a.alloc(30)
    s2 = a.alloc(30)
    s3 = a.alloc(30)
    assert (s1, s2, s3) == (0, 30, 60) and a.largest_free == 10
    assert a.alloc(11) is None
    a.free(s2, 30)
    assert a.alloc(31) is None and a.largest_free == 30
    a.free(s1, 30)  # coalesces with the hole at 30
    assert a.largest_free == 60 and a.free_list == [(0, 60), (90, 10)]
    assert a.alloc(50) == 0 and a.free_list == [(50, 10), (90, 10)]
    a.free(0, 50)
    a.free(s3, 30)
    assert a.free_list == [(0, 100)] and a.free_total == 100


def test_segment_allocator_random_ops_keep_invariants():
    rng = np.random.default_rng(0)
    a = SegmentAllocator(1000)
    live = {}
    for _ in range(2000):
        if live and rng.random() < 0.5:
            s = list(live)[int(rng.integers(len(live)))]
            a.free(s, live.pop(s))
        else:
            n = int(rng.integers(1, 120))
            s = a.alloc(n)
            if s is not None:
                assert all(s + n <= t or t + m <= s for t, m in live.items())  # no overlap
                live[s] = n
        assert a.free_total + sum(live.values()) == 1000
        fl = a.free_list
        assert all(fl[i][0] + fl[i][1] < fl[i + 1][0] for i in range(len(fl) - 1))  # sorted, coalesced


def test_request_validation():
    z = np.zeros(3)
    with pytest.raises(ValueError):
        ReleaseRequest(z, z, z, "euler", 60.0, 3600.0)
    with pytest.raises(ValueError):
        ReleaseRequest(z, z, z, "rk2", 0.0, 3600.0)
    r = ReleaseRequest(z, z, z, "ab3", 120.0, 7200.0, arrival=1.0)
    assert len(r) == 3 and r.latency is None
