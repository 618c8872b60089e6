"""The serving loop's host logic on the CPU (geneva_b200/serve.py), with a
stand-in for the native session (gva_session_*) and for mining: requests are
planned by the real planner, admitted by slots and memory budget, joined to
the running batch between rounds, and each result goes back to its own
request; bad query texts fail alone; closing the server cancels queued
mining requests and stops the running one.
"""
import ctypes
import threading
import time

import pytest

import geneva_b200 as gv
from geneva_b200 import serve

Q3 = "v 0 1\nv 1 2\nv 2 1\ne 0 1 1\ne 1 2 1\n"
Q4 = "v 0 1\nv 1 2\nv 2 1\nv 3 2\ne 0 1 1\ne 1 2 1\ne 2 3 1\n"


class FakeSession:
    """gva_session_* over plain Python: a submitted plan completes after
    `rounds_needed` rounds with count = 1000 + its tag and support = tag % 7."""

    def __init__(self, rounds_needed=2):
        self.rounds_needed = rounds_needed
        self.inflight = {}  # tag -> rounds done
        self.done = []
        self.max_inflight = 0
        self.submits = []
        self.created = None
        self.freed = False
        self.lock = threading.Lock()
        for name in ("gva_session_create", "gva_session_submit", "gva_session_round", "gva_session_poll",
                     "gva_session_free", "gva_last_error"):
            fn = getattr(self, "_" + name)
            setattr(self, name, _Fn(fn))

    def _gva_session_create(self, db, stream, budget, slots, out):
        self.created = (budget, slots)
        out._obj.value = 0x1234
        return 0

    def _gva_session_submit(self, ses, plans, tags, n):
        with self.lock:
            self.submits.append([int(tags[i]) for i in range(n)])
            for i in range(n):
                self.inflight[int(tags[i])] = 0
            self.max_inflight = max(self.max_inflight, len(self.inflight))
        return 0

    def _gva_session_round(self, ses, active):
        with self.lock:
            for t in list(self.inflight):
                self.inflight[t] += 1
                if self.inflight[t] >= self.rounds_needed:
                    del self.inflight[t]
                    self.done.append(t)
            active._obj.value = len(self.inflight)
        return 0

    def _gva_session_poll(self, ses, tags, counts, sups, cap):
        with self.lock:
            n = min(cap, len(self.done))
            for i in range(n):
                t = self.done.pop(0)
                tags[i], counts[i], sups[i] = t, 1000 + t, t % 7
        return n

    def _gva_session_free(self, ses):
        self.freed = True

    def _gva_last_error(self):
        return b"fake"


class _Fn:
    """A callable that accepts ctypes' argtypes/restype attributes."""

    def __init__(self, fn):
        self.fn = fn

    def __call__(self, *a):
        return self.fn(*a)


class FakeDb:
    def __init__(self, max_vertex_id=4000, num_graphs=10):
        self._h = ctypes.c_void_p(1)
        self.num_graphs = num_graphs
        self._max = max_vertex_id

    def info(self):
        return {"max_vertex_id": self._max}


@pytest.fixture
def fake(monkeypatch, native):
    sess = FakeSession()
    monkeypatch.setattr(serve, "library", lambda: sess)
    return sess


def test_results_go_to_their_requests(fake):
    srv = serve.Server(FakeDb(), budget_bytes=1 << 40, slots=64)
    reqs = [srv.submit_match(Q3 if i % 2 else Q4) for i in range(40)]
    res = [r.future.result(timeout=30) for r in reqs]
    srv.close()
    # tags are handed out in admission order, which is arrival order here
    assert [c for c, _ in res] == [1000 + i + 1 for i in range(40)]
    assert [s for _, s in res] == [(i + 1) % 7 for i in range(40)]
    assert all(r.done >= r.admitted >= r.arrival for r in reqs)
    assert fake.freed and fake.created == (1 << 40, 64)


def test_slots_bound_the_requests_in_flight(fake):
    srv = serve.Server(FakeDb(), budget_bytes=1 << 40, slots=4)
    reqs = [srv.submit_match(Q3) for _ in range(30)]
    for r in reqs:
        r.future.result(timeout=30)
    srv.close()
    assert fake.max_inflight <= 4
    assert sum(len(s) for s in fake.submits) == 30


def test_budget_bounds_the_reserved_memory(fake):
    db = FakeDb(max_vertex_id=4000)
    est = 4 * 4 * (4000 // 4 + 1)  # a 4-vertex query's estimate
    srv = serve.Server(db, budget_bytes=2 * est, slots=64)
    seen = []
    orig = fake._gva_session_submit

    def watch(*a):
        seen.append(srv._reserved)
        return orig(*a)

    fake.gva_session_submit = _Fn(watch)
    reqs = [srv.submit_match(Q4) for _ in range(12)]
    for r in reqs:
        r.future.result(timeout=30)
    srv.close()
    assert max(seen) <= 2 * est  # never more than the budget reserved at a submit
    assert max(len(s) for s in fake.submits) <= 2


def test_a_bad_query_fails_alone(fake):
    srv = serve.Server(FakeDb(), budget_bytes=1 << 40, slots=64)
    good1 = srv.submit_match(Q3)
    bad = srv.submit_match("v 0 1\nv 1 1\n")  # no edges
    good2 = srv.submit_match(Q4)
    assert good1.future.result(timeout=30)[0] > 1000
    assert good2.future.result(timeout=30)[0] > 1000
    with pytest.raises(gv.GenevaError):
        bad.future.result(timeout=30)
    srv.close()


def test_close_cancels_mining(fake, monkeypatch):
    started = threading.Event()
    seen_cancel = []

    def fake_mine(db, max_edges, min_support, stream=None, cancel=None, **kw):
        started.set()
        while not cancel.value:  # a running mining request stops once the server closes
            time.sleep(0.001)
        seen_cancel.append(cancel.value)
        raise gv.GenevaError(7, "cancelled")

    monkeypatch.setattr(serve, "mine", fake_mine)
    srv = serve.Server(FakeDb(), budget_bytes=1 << 40, slots=64)
    running = srv.submit_mine(3, 10)
    assert started.wait(10)
    queued = srv.submit_mine(3, 10)
    srv.close()
    with pytest.raises(gv.GenevaError):
        running.future.result(timeout=10)
    with pytest.raises(gv.GenevaError, match="closed"):
        queued.future.result(timeout=10)
    assert seen_cancel == [1]


def test_mining_admission_rejects_beyond_the_queue_limit(fake, monkeypatch):
    """At most mine_queue_limit mining requests wait behind the running one;
    later ones are rejected at arrival (status REJECTED) and the admitted ones
    all complete."""
    release = threading.Event()
    started = threading.Event()

    def fake_mine(db, max_edges, min_support, stream=None, cancel=None, **kw):
        started.set()
        release.wait(10)
        return ("patterns", {"candidates": max_edges})

    monkeypatch.setattr(serve, "mine", fake_mine)
    srv = serve.Server(FakeDb(), budget_bytes=1 << 40, slots=64, mine_queue_limit=2)
    first = srv.submit_mine(3, 10)
    assert started.wait(10)  # running, no longer queued
    reqs = [srv.submit_mine(4, 10) for _ in range(6)]
    rejected = [r for r in reqs if r.future.done()]
    assert len(rejected) == 4 and srv.mine_rejected == 4
    for r in rejected:
        with pytest.raises(gv.GenevaError) as e:
            r.future.result(timeout=1)
        assert e.value.status == serve.REJECTED
    release.set()
    assert first.future.result(timeout=10)[1]["candidates"] == 3
    for r in reqs:
        if r not in rejected:
            assert r.future.result(timeout=10)[1]["candidates"] == 4
    srv.close()
