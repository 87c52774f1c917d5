"""Host logic of the serving loop (cuhepy_b200.serving.Scheduler), no GPU:
admission by lanes and memory, FIFO order, merging, errors, release."""

import threading
import time

import pytest

from cuhepy_b200.serving import Request, Scheduler


class Gate:
    """Fake executor whose groups block until opened; records what ran."""

    def __init__(self):
        self.groups = []
        self.events = []
        self.lock = threading.Lock()

    def __call__(self, kind, index, group, lane, deliver=None):
        ev = threading.Event()
        with self.lock:
            self.groups.append(([r.seq for r in group], lane))
            self.events.append(ev)
        assert ev.wait(10)
        if any(r.payload == "boom" for r in group):
            raise RuntimeError("executor failed")
        return [("answer", r.payload) for r in group]

    def open(self, k):
        deadline = time.time() + 10
        while len(self.events) <= k:
            assert time.time() < deadline
            time.sleep(0.001)
        self.events[k].set()

    def wait_groups(self, count):
        deadline = time.time() + 10
        while len(self.groups) < count:
            assert time.time() < deadline
            time.sleep(0.001)


def _req(kind="paillier", index="a", queries=1, nbytes=10, payload=None):
    return Request(kind, index, queries, nbytes, payload)


def test_memory_admission_and_release():
    gate = Gate()
    s = Scheduler(gate, lanes=4, budget_bytes=100)
    s.start()
    try:
        f1 = s.submit(_req(nbytes=60, payload=1))
        gate.wait_groups(1)
        f2 = s.submit(_req(index="b", nbytes=60, payload=2))
        time.sleep(0.05)
        assert len(gate.groups) == 1          # 60 + 60 > 100: waits although lanes are free
        gate.open(0)
        assert f1.result(5) == ("answer", 1)
        time.sleep(0.05)
        assert len(gate.groups) == 1          # the answer still holds its bytes
        s.release(60)
        gate.wait_groups(2)
        gate.open(1)
        assert f2.result(5) == ("answer", 2)
        s.release(60)
        assert s.in_use == 0 and s.peak_in_use <= 100
    finally:
        for e in gate.events:
            e.set()
        s.stop()


def test_waiting_requests_of_one_index_are_merged_up_to_max_batch():
    gate = Gate()
    s = Scheduler(gate, lanes={"paillier": 1, "bfv": 1}, budget_bytes=10_000, max_batch=8)
    s.start()
    try:
        first = s.submit(_req(queries=1, payload="x"))
        gate.wait_groups(1)                    # the only Paillier lane is busy from here on
        futs = [s.submit(_req(queries=3, payload=i)) for i in range(4)]
        other = s.submit(_req(index="b", queries=1, payload="b"))
        gate.open(0)
        gate.wait_groups(2)
        # head (3) + next (3) fit 8; the third would make 9; "b" is another index
        assert gate.groups[1][0] == [1, 2]
        gate.open(1)
        gate.wait_groups(3)
        assert gate.groups[2][0] == [3, 4]
        gate.open(2)
        gate.wait_groups(4)
        assert gate.groups[3][0] == [5]
        gate.open(3)
        assert [f.result(5) for f in futs] == [("answer", i) for i in range(4)]
        assert other.result(5) == ("answer", "b")
        assert first.result(5) == ("answer", "x")
        # BFV requests are never merged: each is its own launch
        bfv = [s.submit(_req(kind="bfv", index="a", queries=1, nbytes=0, payload=f"q{i}")) for i in range(2)]
        gate.wait_groups(5)
        gate.open(4)
        gate.wait_groups(6)
        gate.open(5)
        assert [f.result(5) for f in bfv] == [("answer", "q0"), ("answer", "q1")]
        assert [len(g) for g, _ in gate.groups[4:]] == [1, 1]
    finally:
        for e in gate.events:
            e.set()
        s.stop()


def test_fifo_head_is_not_overtaken():
    gate = Gate()
    s = Scheduler(gate, lanes=3, budget_bytes=100)
    s.start()
    try:
        s.submit(_req(index="a", nbytes=50, payload=0))
        gate.wait_groups(1)
        big_req = _req(index="b", nbytes=80, payload=1)      # does not fit yet
        small_req = _req(index="c", nbytes=10, payload=2)    # would fit, must wait behind
        big, small = s.submit(big_req), s.submit(small_req)
        time.sleep(0.05)
        assert len(gate.groups) == 1
        gate.open(0)
        s.release(50)
        gate.wait_groups(3)            # 80 + 10 <= 100: both run once the head fits
        assert sorted(g for g, _ in gate.groups[1:]) == [[1], [2]]
        assert big_req.admitted <= small_req.admitted
        gate.open(1)
        gate.open(2)
        assert big.result(5) == ("answer", 1) and small.result(5) == ("answer", 2)
    finally:
        for e in gate.events:
            e.set()
        s.stop()


def test_oversize_requests_are_refused_and_errors_reach_every_caller():
    gate = Gate()
    s = Scheduler(gate, lanes=2, budget_bytes=100, max_batch=4)
    s.start()
    try:
        with pytest.raises(MemoryError):
            s.submit(_req(nbytes=101))
        with pytest.raises(ValueError):
            s.submit(_req(queries=5))
        blocker = s.submit(_req(index="z", payload="z"))
        gate.wait_groups(1)
        blocker2 = s.submit(_req(index="y", payload="y"))
        gate.wait_groups(2)
        f1 = s.submit(_req(payload="boom"))
        f2 = s.submit(_req(payload="fine"))
        gate.open(0)
        gate.wait_groups(3)
        gate.open(2)
        for f in (f1, f2):                     # merged with the failing request
            with pytest.raises(RuntimeError, match="executor failed"):
                f.result(5)
        gate.open(1)
        blocker.result(5)
        blocker2.result(5)
        s.release(20)
        assert s.in_use == 0                   # failed requests freed their bytes
    finally:
        for e in gate.events:
            e.set()
        s.stop()


def test_lanes_bound_concurrency():
    running = []
    peak = [0]
    lock = threading.Lock()

    def execute(kind, index, group, lane, deliver):
        with lock:
            running.append(lane)
            peak[0] = max(peak[0], len(running))
        time.sleep(0.02)
        with lock:
            running.remove(lane)
        return [r.payload for r in group]

    s = Scheduler(execute, lanes=3, budget_bytes=10**9, holds_memory=lambda kind: False)
    s.start()
    try:
        futs = [s.submit(_req(kind="bfv", index=str(i), nbytes=0, payload=i)) for i in range(12)]
        assert [f.result(5) for f in futs] == list(range(12))
        assert peak[0] == 3 and s.max_concurrent == 3
        assert s.in_use == 0
    finally:
        s.stop()


def test_stop_resolves_waiting_requests():
    def execute(kind, index, group, lane, deliver):
        time.sleep(0.05)
        return [r.payload for r in group]

    s = Scheduler(execute, lanes=1, budget_bytes=100, holds_memory=lambda kind: False)
    s.start()
    first = s.submit(_req(payload=0))
    waiting = s.submit(_req(index="b", payload=1))
    s.stop()
    assert first.done() and waiting.done()
    assert waiting.exception() is None or isinstance(waiting.exception(), RuntimeError)
    with pytest.raises(RuntimeError):
        s.submit(_req())


def test_kinds_do_not_wait_for_each_other_and_answers_can_come_early():
    gate = Gate()
    order = []

    def execute(kind, index, group, lane, deliver):
        if kind == "paillier":
            return gate(kind, index, group, lane)
        for k, r in enumerate(group):
            deliver(k, ("early", r.payload))
            order.append(r.payload)
        return [None] * len(group)

    s = Scheduler(execute, lanes={"paillier": 1, "bfv": 2}, budget_bytes=100)
    s.start()
    try:
        p1 = s.submit(_req(nbytes=90, payload="p1"))
        gate.wait_groups(1)
        p2 = s.submit(_req(index="b", nbytes=50, payload="p2"))   # blocked by memory
        b = [s.submit(_req(kind="bfv", index="x", nbytes=0, payload=i)) for i in range(3)]
        assert [f.result(5) for f in b] == [("early", i) for i in range(3)]
        assert not p2.done()
        gate.open(0)
        assert p1.result(5) == ("answer", "p1")
        s.release(90)
        gate.wait_groups(2)
        gate.open(1)
        assert p2.result(5) == ("answer", "p2")
        assert s.lane_ids("paillier") == [0] and s.lane_ids("bfv") == [1, 2]
    finally:
        for e in gate.events:
            e.set()
        s.stop()


def test_shortest_first_with_aging():
    """The serving policy for Paillier requests: the fewest queries go first,
    but a request that has waited past the age limit is not overtaken."""
    from cuhepy_b200.serving import shortest_first

    gate = Gate()
    s = Scheduler(gate, lanes=1, budget_bytes=1000, merge=lambda kind: False, pick=shortest_first(0.5))
    s.start()
    try:
        s.submit(_req(queries=1, payload="running"))
        gate.wait_groups(1)
        reqs = {name: _req(queries=q, payload=name) for name, q in (("big", 40), ("mid", 9), ("small", 2))}
        futs = {name: s.submit(r) for name, r in reqs.items()}
        time.sleep(0.05)
        for k in range(4):
            gate.open(k)
            if k < 3:
                gate.wait_groups(k + 2)
        assert [futs[name].result(5)[1] for name in ("small", "mid", "big")] == ["small", "mid", "big"]
        assert reqs["small"].admitted < reqs["mid"].admitted < reqs["big"].admitted
        # aged: the oldest waiting request goes first once past the limit
        s.submit(_req(queries=1, payload="running2"))
        gate.wait_groups(5)
        old_req, young_req = _req(queries=50, payload="old"), _req(queries=1, payload="young")
        old = s.submit(old_req)
        time.sleep(0.6)
        young = s.submit(young_req)
        gate.open(4)
        gate.wait_groups(6)
        gate.open(5)
        gate.wait_groups(7)
        gate.open(6)
        assert old.result(5)[1] == "old" and young.result(5)[1] == "young"
        assert old_req.admitted < young_req.admitted
    finally:
        for e in gate.events:
            e.set()
        s.stop()


def test_overtaking_never_starves_the_oldest_of_memory():
    """Shortest-first admission with answers that hold their memory: a small
    request may overtake the oldest only while the oldest still fits, so a
    caller reading answers in submission order is never blocked."""
    from cuhepy_b200.serving import shortest_first

    gate = Gate()
    s = Scheduler(gate, lanes=2, budget_bytes=100, merge=lambda kind: False, pick=shortest_first(10.0))
    s.start()
    try:
        s.submit(_req(queries=1, nbytes=30, payload="first"))
        gate.wait_groups(1)
        old_req = _req(queries=8, nbytes=60, payload="old")      # fits (30 + 60 <= 100) only alone
        small_req = _req(queries=1, nbytes=20, payload="small")  # would leave 50 < 60: must not overtake
        old, small = s.submit(old_req), s.submit(small_req)
        gate.wait_groups(2)
        assert old_req.admitted and not small_req.admitted
        gate.open(0)
        gate.open(1)
        assert old.result(5)[1] == "old"
        s.release(30)
        s.release(60)
        gate.open(2)
        assert small.result(5)[1] == "small"
    finally:
        for e in gate.events:
            e.set()
        s.stop()
