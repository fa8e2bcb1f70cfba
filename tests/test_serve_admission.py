"""Host logic of the served form's admission (no GPU): large requests run
alone, small ones are packed in arrival order under the budget, the batch
size and the per-batch NIP cap; unsized requests stop the scan."""
import threading
from collections import deque

import pytest

from gpuspgemm_b200.serve import Request, SpgemmServer


def _server(**kw):
    s = SpgemmServer.__new__(SpgemmServer)  # admission state only; no handles
    s.memory_budget = kw.get("memory_budget", 1 << 40)
    s.max_batch = kw.get("max_batch", 256)
    s.solo_nip = kw.get("solo_nip", 1000)
    s.batch_nip = kw.get("batch_nip", 5000)
    s.batch_nip_min = kw.get("batch_nip_min", s.batch_nip)
    s.batch_cols = kw.get("batch_cols", 1 << 40)
    s.workers = kw.get("workers", 1)
    s._queue = deque()
    s._in_flight_bytes = 0
    s._cv = threading.Condition()
    return s


class _Op:
    def __init__(self, n):
        self.n = n


def _req(rid, nip, bound=None, cols=10):
    r = Request(None, _Op(cols), rid=rid)
    r.nip = nip
    r.bound_bytes = nip * 12 if bound is None else bound
    return r


def _ids(rs):
    return [r.rid for r in rs]


def test_large_alone_small_packed_in_order():
    s = _server()
    s._queue.extend([_req(0, 10), _req(1, 2000), _req(2, 20), _req(3, 30), _req(4, 5000)])
    taken, solo = s._admit()
    assert _ids(taken) == [0, 2, 3] and not solo
    assert _ids(s._queue) == [1, 4]            # large ones keep their order
    taken, solo = s._admit()
    assert _ids(taken) == [1] and solo
    taken, solo = s._admit()
    assert _ids(taken) == [4] and solo
    assert not s._queue


def test_batch_nip_cap_and_max_batch():
    s = _server(batch_nip=100, max_batch=3)
    s._queue.extend([_req(i, 40) for i in range(6)])
    assert _ids(s._admit()[0]) == [0, 1]       # 40 + 40 + 40 > 100
    s = _server(batch_nip=10_000, max_batch=3)
    s._queue.extend([_req(i, 40) for i in range(6)])
    assert _ids(s._admit()[0]) == [0, 1, 2]


def test_budget_and_oversize_request():
    s = _server(memory_budget=1000)
    s._queue.extend([_req(0, 10, 600), _req(1, 10, 600), _req(2, 10, 5000)])
    assert _ids(s._admit()[0]) == [0]          # the second does not fit beside it
    assert s._in_flight_bytes == 600
    assert s._admit()[0] == []                 # nothing fits while 0 is in flight
    s._in_flight_bytes = 0
    assert _ids(s._admit()[0]) == [1]
    s._in_flight_bytes = 0
    assert _ids(s._admit()[0]) == [2]          # larger than the budget: alone, when idle


def test_unsized_request_stops_the_scan():
    s = _server()
    s._queue.extend([_req(0, 10), _req(1, 10, bound=-1), _req(2, 10)])
    assert _ids(s._admit()[0]) == [0]
    assert _ids(s._queue) == [1, 2]


@pytest.mark.parametrize("n", [1, 7])
def test_skipped_large_requests_are_restored(n):
    s = _server(max_batch=2)
    s._queue.extend([_req(0, 10)] + [_req(10 + i, 4000) for i in range(n)] + [_req(1, 10),
                                                                              _req(2, 10)])
    assert _ids(s._admit()[0]) == [0, 1]
    assert _ids(s._queue) == [10 + i for i in range(n)] + [2]


def test_batch_cap_follows_the_backlog():
    # a long queue makes long batches (up to batch_nip), a short one short ones
    s = _server(batch_nip=1000, batch_nip_min=100, workers=2)
    s._queue.extend([_req(i, 40) for i in range(100)])      # backlog 4000 -> cap 1000
    assert len(s._admit()[0]) == 25
    s = _server(batch_nip=1000, batch_nip_min=100, workers=2)
    s._queue.extend([_req(i, 40) for i in range(6)])        # backlog 240 -> cap 120
    assert len(s._admit()[0]) == 3


def test_batch_column_cap():
    s = _server(batch_cols=100)
    s._queue.extend([_req(i, 10, cols=40) for i in range(5)])
    assert _ids(s._admit()[0]) == [0, 1]
    s = _server(batch_cols=100)
    s._queue.extend([_req(0, 10, cols=500), _req(1, 10, cols=5)])
    assert _ids(s._admit()[0]) == [0]           # wider than the cap: alone

