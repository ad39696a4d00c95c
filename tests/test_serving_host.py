"""Host-side scheduling of the search server (no GPU): admission by HBM budget, one request per
scene in flight, arrival order kept per scene."""
import collections
import threading

from torchcompactradius_b200.serving import Request, SearchServer


class FakeScene:
    def __init__(self, nbytes):
        self.nbytes = nbytes

    def bytes_estimate(self):
        return self.nbytes


def _server(sizes, budget, max_batch=64):
    s = SearchServer.__new__(SearchServer)
    s.scenes = [FakeScene(b) for b in sizes]
    s.hbm_budget = budget
    s.max_batch = max_batch
    s._pending = collections.deque()
    s._busy = set()
    s._in_use = 0
    s._cv = threading.Condition()
    return s


def test_admission_respects_the_budget_and_arrival_order():
    s = _server([10, 20, 30, 40], budget=60)
    for k in (0, 1, 2, 3):
        s._pending.append(Request(k, arrival=float(k)))
    first = s._admit()
    assert [r.scene for r in first] == [0, 1, 2]  # 60 bytes: scene 3 waits for memory
    assert s._in_use == 60 and s._busy == {0, 1, 2}
    assert [r.scene for r in s._pending] == [3]
    assert s._admit() == []  # nothing fits until memory frees up
    s._in_use -= 30  # scene 2 done: 30 + 40 still exceeds 60
    s._busy.discard(2)
    assert s._admit() == []
    s._in_use -= 20  # scene 1 done
    s._busy.discard(1)
    assert [r.scene for r in s._admit()] == [3]


def test_one_request_per_scene_in_flight_and_per_scene_order():
    s = _server([5, 5], budget=100)
    reqs = [Request(0, arrival=0.0), Request(0, arrival=1.0), Request(1, arrival=2.0), Request(0, arrival=3.0)]
    s._pending.extend(reqs)
    a = s._admit()
    assert a == [reqs[0], reqs[2]]
    assert list(s._pending) == [reqs[1], reqs[3]]
    s._busy.discard(0)
    s._in_use -= 5
    b = s._admit()
    assert b == [reqs[1]]  # the scene's next request, not the one after it
    s._busy.discard(0)
    assert s._admit() == [reqs[3]]


def test_a_request_held_back_blocks_later_requests_of_its_scene():
    s = _server([50, 5], budget=54)
    s._in_use = 0
    reqs = [Request(1), Request(0), Request(1)]
    s._pending.extend(reqs)
    a = s._admit()
    assert a == [reqs[0]]  # scene 0 does not fit next to it; scene 1's second request stays behind its first
    assert list(s._pending) == [reqs[1], reqs[2]]


def test_max_batch_limits_a_group():
    s = _server([1] * 10, budget=1000, max_batch=4)
    s._pending.extend(Request(k) for k in range(10))
    assert len(s._admit()) == 4
    assert len(s._admit()) == 4
    assert len(s._admit()) == 2
