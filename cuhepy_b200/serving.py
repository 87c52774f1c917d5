"""Encrypted kNN request loop on one B200: resident indexes, continuous batching.

A :class:`KnnEvaluator` keeps encrypted indexes and evaluation keys resident
in HBM and answers two kinds of request:

* Paillier-Lookup (``submit_paillier``): B encrypted query vectors of
  ``chunk_num`` chunk ciphertexts each.  The answer is encode_hamming_server
  of every query with every index vector, chunk by chunk
  (``hamming/paillier_lookup.py:362-370`` of the reference: one product mod
  n^2 per chunk), as a device tensor ``[chunk_num, B, V, K]`` of u32 limbs.
* BFV (``submit_bfv``): one packed query ciphertext against a resident packed
  index; the answer is the list of packed response ciphertexts of
  ``packed_search`` (``bfv/_cpu_ext/bindings.cpp:329-367``).

Continuous batching.  Requests wait in one queue per kind.  A scheduler
thread admits a request of a kind as soon as one of that kind's execution
lanes is free and the device memory the request needs fits in the budget
(free HBM at start minus a reserve and the BFV lanes' workspaces).  Admitted
work runs on the lane's own CUDA stream, so requests that arrive while
others are on the GPU overlap with them.  BFV searches are chains of short
kernels and run concurrently on several lanes whose streams have the
highest priority, so their blocks are scheduled ahead of queued Paillier
blocks; they are admitted in arrival order.  Paillier work saturates the GPU
by itself (one query against a million vectors is a million products): it
gets one lane fed in arrival order by default.  With ``age_limit_s`` > 0 the
waiting request with the fewest queries goes next (shortest job first)
unless the oldest has waited longer than that, and only while the oldest
still fits in memory; with ``paillier_lanes`` > 1 requests share the GPU
block by block.  (On the bench's 80%-load trace both lowered the median
Paillier latency less than they raised its tail, so neither is the
default.)  Paillier requests on a small index
(a launch over one query would not fill the GPU) that are waiting when a
lane frees up are merged into one launch (up to ``max_batch`` queries).
The memory of a Paillier answer stays reserved until the caller releases
the result; a request larger than the whole budget is refused at
submission.

``run_plain`` is the comparison point: one request at a time, one launch per
query, every launch waited for.

The scheduler logic is independent of the GPU (executors are pluggable), so
it is tested on the host with fake executors.
"""

from __future__ import annotations

import collections
import itertools
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Any, Callable


@dataclass
class Request:
    """One queued request (scheduler view)."""

    kind: str            # "paillier" or "bfv"
    index: str           # name of the resident index
    queries: int         # query vectors carried (merging unit)
    nbytes: int          # device bytes held while the answer is alive
    payload: Any
    arrival: float = field(default_factory=time.perf_counter)
    admitted: float = 0.0
    finished: float = 0.0
    future: Future = field(default_factory=Future)
    seq: int = 0
    lane: int = -1


class Scheduler:
    """Admission by free lanes and device memory, FIFO per request kind, with
    request merging.

    ``lanes`` maps each request kind to its number of execution lanes; the
    kinds do not wait for each other (bulk Paillier work on its lane, BFV
    searches on theirs), and within a kind requests are admitted oldest
    first.  ``execute(kind, index, requests, lane, deliver)`` runs one
    admitted group; it may hand over an answer early with
    ``deliver(position, answer)`` and returns the answers it did not deliver
    (one per request, in order; delivered positions are ignored).
    ``holds_memory(kind)`` says whether an answer keeps its bytes reserved
    until ``release`` (True) or frees them at completion (False).
    """

    def __init__(self, execute: Callable[..., list[Any]], lanes: dict[str, int] | int,
                 budget_bytes: int, max_batch: int = 64,
                 holds_memory: Callable[[str], bool] = lambda kind: True,
                 merge: Callable[[str], bool] = lambda kind: kind == "paillier",
                 mergeable: Callable[[Request], bool] = lambda req: True,
                 pick: Callable[[str, Any, float, int], int] | None = None) -> None:
        if isinstance(lanes, int):
            lanes = {"paillier": lanes, "bfv": lanes}
        if not lanes or min(lanes.values()) < 1:
            raise ValueError("at least one lane per request kind")
        self._execute = execute
        self._holds = holds_memory
        self._merge = merge
        self._mergeable = mergeable
        self._pick = pick or (lambda kind, queue, now, free: 0)
        self.lanes = dict(lanes)
        self.budget = int(budget_bytes)
        self.max_batch = int(max_batch)
        self.in_use = 0
        self.peak_in_use = 0
        # lane ids are global: kind k owns a contiguous range
        self._lane_kind: list[str] = []
        self._free: dict[str, list[int]] = {}
        for kind, count in self.lanes.items():
            ids = list(range(len(self._lane_kind), len(self._lane_kind) + count))
            self._lane_kind += [kind] * count
            self._free[kind] = ids
        self._queues: dict[str, collections.deque[Request]] = {k: collections.deque() for k in self.lanes}
        self._cv = threading.Condition()
        self._seq = itertools.count()
        self._running = False
        self._thread: threading.Thread | None = None
        self._workers: list[threading.Thread] = []
        total = len(self._lane_kind)
        self._work: list[collections.deque] = [collections.deque() for _ in range(total)]
        self._work_cv = [threading.Condition() for _ in range(total)]
        self.completed: list[Request] = []
        self.launches = 0
        self.max_concurrent = 0
        self._busy = 0

    def lane_ids(self, kind: str) -> list[int]:
        return [i for i, k in enumerate(self._lane_kind) if k == kind]

    # -- lifetime -----------------------------------------------------------
    def start(self) -> None:
        with self._cv:
            if self._running:
                return
            self._running = True
        for lane in range(len(self._lane_kind)):
            t = threading.Thread(target=self._worker, args=(lane,), name=f"knn-lane-{lane}", daemon=True)
            t.start()
            self._workers.append(t)
        self._thread = threading.Thread(target=self._loop, name="knn-scheduler", daemon=True)
        self._thread.start()

    def stop(self) -> None:
        with self._cv:
            self._running = False
            self._cv.notify_all()
        if self._thread:
            self._thread.join()  # no dispatch can follow the sentinels below
        for lane, cv in enumerate(self._work_cv):
            with cv:
                self._work[lane].append(None)
                cv.notify()
        for t in self._workers:
            t.join()
        self._workers.clear()
        with self._cv:
            for q in self._queues.values():
                while q:
                    q.popleft().future.set_exception(RuntimeError("evaluator stopped"))

    # -- submission ---------------------------------------------------------
    def submit(self, req: Request) -> Future:
        if req.kind not in self._queues:
            raise ValueError(f"no lanes for request kind {req.kind!r}")
        if req.nbytes > self.budget:
            raise MemoryError(f"request needs {req.nbytes} device bytes; the budget is {self.budget}")
        if req.queries > self.max_batch and self._merge(req.kind):
            raise ValueError(f"at most {self.max_batch} queries per request")
        with self._cv:
            if not self._running:
                raise RuntimeError("evaluator is not running")
            req.seq = next(self._seq)
            self._queues[req.kind].append(req)
            self._cv.notify_all()
        return req.future

    def release(self, nbytes: int) -> None:
        with self._cv:
            self.in_use -= int(nbytes)
            self._cv.notify_all()

    # -- scheduling ---------------------------------------------------------
    def _admit(self) -> tuple[list[Request], int] | None:
        """The head request of a kind with a free lane (the oldest, unless
        the ``pick`` policy names another), if its memory fits; later
        requests of the same index join it while the group stays within
        max_batch queries and the budget."""
        now = time.perf_counter()
        for kind, queue in self._queues.items():
            if not queue or not self._free[kind]:
                continue
            at = self._pick(kind, queue, now, self.budget - self.in_use)
            head = queue[at]
            if self.in_use + head.nbytes > self.budget:
                continue
            del queue[at]
            group = [head]
            need = head.nbytes
            if self._merge(kind) and self._mergeable(head):
                total = head.queries
                keep: collections.deque[Request] = collections.deque()
                while queue:
                    r = queue.popleft()
                    if (r.index == head.index and self._mergeable(r) and total + r.queries <= self.max_batch
                            and self.in_use + need + r.nbytes <= self.budget):
                        group.append(r)
                        total += r.queries
                        need += r.nbytes
                    else:
                        keep.append(r)
                self._queues[kind] = keep
            lane = self._free[kind].pop(0)
            self.in_use += need
            self.peak_in_use = max(self.peak_in_use, self.in_use)
            return group, lane
        return None

    def _loop(self) -> None:
        while True:
            with self._cv:
                picked = None
                while self._running and picked is None:
                    picked = self._admit()
                    if picked is None:
                        self._cv.wait()
                if not self._running:
                    return
                group, lane = picked
                now = time.perf_counter()
                for r in group:
                    r.admitted = now
                    r.lane = lane
                self._busy += 1
                self.max_concurrent = max(self.max_concurrent, self._busy)
            with self._work_cv[lane]:
                self._work[lane].append(group)
                self._work_cv[lane].notify()

    def _finish(self, req: Request, answer: Any = None, error: BaseException | None = None) -> None:
        now = time.perf_counter()
        with self._cv:
            req.finished = now
            if error is not None or not self._holds(req.kind):
                self.in_use -= req.nbytes
            self.completed.append(req)
            self._cv.notify_all()
        if error is not None:
            req.future.set_exception(error)
        else:
            req.future.set_result(answer)

    def _worker(self, lane: int) -> None:
        while True:
            with self._work_cv[lane]:
                while not self._work[lane]:
                    self._work_cv[lane].wait()
                group = self._work[lane].popleft()
            if group is None:
                return
            kind, index = group[0].kind, group[0].index
            delivered = [False] * len(group)

            def deliver(k: int, answer: Any) -> None:
                if not delivered[k]:
                    delivered[k] = True
                    self._finish(group[k], answer)

            try:
                answers = self._execute(kind, index, group, lane, deliver)
                error = None
            except BaseException as exc:  # noqa: BLE001 - delivered to every waiting caller
                answers, error = None, exc
            for k, r in enumerate(group):
                if not delivered[k]:
                    delivered[k] = True
                    self._finish(r, None if error else answers[k], error)
            with self._cv:
                self.launches += 1
                self._busy -= 1
                self._free[kind].append(lane)
                self._free[kind].sort()
                self._cv.notify_all()


def shortest_first(age_limit_s: float) -> Callable[[str, Any, float, int], int]:
    """A ``pick`` policy for :class:`Scheduler`: the waiting request with the
    fewest queries (the earliest among equals), unless the oldest request has
    waited longer than ``age_limit_s``, which then goes first.  A request may
    overtake the oldest only if the oldest still fits in the free memory
    after it, so an overtaking answer (whose memory stays reserved until its
    caller releases it) never keeps the oldest request from being admitted:
    a caller that reads its answers in submission order always progresses."""

    def pick(kind: str, queue, now: float, free: int) -> int:
        head = queue[0]
        if len(queue) < 2 or now - head.arrival > age_limit_s or head.nbytes > free:
            return 0
        room = free - head.nbytes
        return min((i for i in range(len(queue)) if i == 0 or queue[i].nbytes <= room),
                   key=lambda i: (queue[i].queries, i))

    return pick


class PaillierAnswer:
    """encode_hamming_server products of one request, on the device:
    ``tensor[c, b, v]`` = query b chunk c times index vector v chunk c mod n^2
    (K little-endian u32 limbs, stored as int32).  ``release()`` returns its
    memory to the evaluator's budget; read the tensor on the device before,
    or synchronise the stream that read it."""

    def __init__(self, tensor, release: Callable[[], None]) -> None:
        self.tensor = tensor
        self._release = release

    def release(self) -> None:
        if self._release is not None:
            self.tensor = None
            fn, self._release = self._release, None
            fn()

    def __del__(self) -> None:  # pragma: no cover - safety net
        try:
            self.release()
        except Exception:
            pass


class KnnEvaluator:
    """Resident-index kNN evaluator on one GPU (see the module docstring)."""

    #: below this many index vectors, waiting Paillier requests are merged
    #: into one launch (a launch over one query would not fill the GPU);
    #: above it, the group's requests run back to back, each delivered as
    #: soon as its own launch ends
    MERGE_BELOW_VECTORS = 1 << 18

    def __init__(self, device: int = 0, paillier_lanes: int = 1, bfv_lanes: int = 3, max_batch: int = 64,
                 reserve_bytes: int = 2 << 30, budget_bytes: int | None = None,
                 age_limit_s: float = 0.0) -> None:
        import torch

        self._torch = torch
        self.device = int(device)
        self.lane_counts = {"paillier": int(paillier_lanes), "bfv": int(bfv_lanes)}
        self.max_batch = int(max_batch)
        self.age_limit_s = float(age_limit_s)
        self.reserve_bytes = int(reserve_bytes)
        self._budget_override = budget_bytes
        # bulk work on default-priority streams; BFV lanes are the ring's own
        # highest-priority streams
        self._streams = [torch.cuda.Stream(device=self.device) for _ in range(self.lane_counts["paillier"])]
        self._paillier: dict[str, dict] = {}
        self._bfv: dict[str, dict] = {}
        self._sched: Scheduler | None = None

    # -- resident state ---------------------------------------------------
    def add_paillier_index(self, name: str, n: int, index) -> None:
        """Keep a Paillier-Lookup encrypted index resident: ``index`` is
        ``[V, chunk_num, K]`` (or ``[V, K]``) u32 limbs as an int32 tensor
        or numpy array; it is copied to the device once."""
        from cuhepy_b200.paillier.gpu import PaillierDevice

        torch = self._torch
        t = torch.as_tensor(index)
        if t.dtype != torch.int32:
            t = t.view(torch.int32) if t.dtype == torch.uint32 else t.to(torch.int32)
        if t.dim() == 2:
            t = t.unsqueeze(1)
        contexts = []
        for lane in range(len(self._streams)):
            ctx = PaillierDevice(int(n), self.device)
            ctx.set_stream(self._streams[lane].cuda_stream)
            contexts.append(ctx)
        words = contexts[0].words
        if t.dim() != 3 or t.shape[2] != words:
            raise ValueError(f"index must be [V, chunk_num, {words}] limbs")
        vectors, chunks = int(t.shape[0]), int(t.shape[1])
        # chunk-major resident layout: [chunk_num, V, K]
        dev = t.to(f"cuda:{self.device}").permute(1, 0, 2).contiguous()
        self._paillier[name] = {"n": int(n), "index": dev, "vectors": vectors, "chunks": chunks,
                                "words": words, "contexts": contexts}

    def add_bfv_index(self, name: str, server, index, count: int, compact: bool = True) -> None:
        """Keep a BFV index resident: ``server`` from ``_bfv_rns.create_server``
        and ``index`` from ``_bfv_rns.upload_index``; ``count`` vectors."""
        from cuhepy_b200.bfv import _bfv_rns

        _bfv_rns.set_lanes(server.ring, self.lane_counts["bfv"])
        # every lane's workspace now: an allocation inside a request would
        # wait for whatever else runs on the GPU
        _bfv_rns.reserve_workspace(server, index.tiles, compact)
        self._bfv[name] = {"server": server, "index": index, "count": int(count), "compact": bool(compact),
                           "workspace": _bfv_rns.search_workspace(server, index.tiles, compact)}

    def paillier_answer_bytes(self, name: str, queries: int) -> int:
        p = self._paillier[name]
        return p["chunks"] * int(queries) * p["vectors"] * p["words"] * 4

    # -- lifetime -----------------------------------------------------------
    def start(self) -> None:
        torch = self._torch
        # BFV lanes keep their search workspace: reserve it up front
        bfv_ws = sum(b["workspace"] for b in self._bfv.values()) * self.lane_counts["bfv"]
        if self._budget_override is not None:
            budget = int(self._budget_override)
        elif getattr(self, "_budget", None) is not None:
            budget = self._budget  # fixed at the first start: later the lanes' workspaces are allocated
        else:
            free, _ = torch.cuda.mem_get_info(self.device)
            cached = torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)
            budget = int(free) + int(cached) - self.reserve_bytes - bfv_ws
            self._budget = budget
        if budget <= 0:
            raise MemoryError("no device memory left for answers after the resident state")
        self._sched = Scheduler(self._execute, self.lane_counts, budget, self.max_batch,
                                holds_memory=lambda kind: kind == "paillier",
                                mergeable=self._mergeable, pick=self._pick)
        self._sched.start()

    def stop(self) -> None:
        if self._sched:
            self._sched.stop()

    def __enter__(self):
        self.start()
        return self

    def __exit__(self, *exc) -> None:
        self.stop()

    @property
    def scheduler(self) -> Scheduler:
        if self._sched is None:
            raise RuntimeError("evaluator not started")
        return self._sched

    # -- requests -----------------------------------------------------------
    def submit_paillier(self, name: str, queries) -> Future:
        """queries: ``[B, chunk_num, K]`` (or ``[B, K]``) encrypted query
        chunks, host or device; the future gives a :class:`PaillierAnswer`."""
        torch = self._torch
        p = self._paillier[name]
        q = torch.as_tensor(queries)
        if q.dtype != torch.int32:
            q = q.view(torch.int32) if q.dtype == torch.uint32 else q.to(torch.int32)
        if q.dim() == 2:
            q = q.unsqueeze(1)
        if q.dim() != 3 or q.shape[1] != p["chunks"] or q.shape[2] != p["words"]:
            raise ValueError(f"queries must be [B, {p['chunks']}, {p['words']}] limbs")
        b = int(q.shape[0])
        if b < 1:
            raise ValueError("empty request")
        req = Request("paillier", name, b, self.paillier_answer_bytes(name, b), q)
        return self.scheduler.submit(req)

    def submit_bfv(self, name: str, query) -> Future:
        """query: the packed (b, a) query ciphertext; the future gives the
        packed response ciphertexts."""
        if name not in self._bfv:
            raise KeyError(name)
        return self.scheduler.submit(Request("bfv", name, 1, 0, query))

    # -- policy -------------------------------------------------------------
    def _mergeable(self, req: Request) -> bool:
        """Requests on small Paillier indexes share one launch; on large ones
        (a launch per query already fills the GPU) each is admitted alone,
        so the next pick happens as soon as a lane frees."""
        return req.kind != "paillier" or self._paillier[req.index]["vectors"] < self.MERGE_BELOW_VECTORS

    def _pick(self, kind: str, queue, now: float, free: int) -> int:
        """Paillier: shortest job first with aging; BFV searches (all of one
        size) in arrival order."""
        return shortest_first(self.age_limit_s)(kind, queue, now, free) if kind == "paillier" else 0

    # -- execution ----------------------------------------------------------
    def _execute(self, kind: str, name: str, group: list[Request], lane: int, deliver) -> list[Any]:
        if kind == "bfv":
            from cuhepy_b200.bfv import _bfv_rns

            b = self._bfv[name]
            return [_bfv_rns.search_index(b["server"], b["index"], r.payload, b["count"], b["compact"])
                    for r in group]
        slot = lane - self.scheduler.lane_ids("paillier")[0]
        p = self._paillier[name]
        if p["vectors"] >= self.MERGE_BELOW_VECTORS and len(group) > 1:
            answers = []
            for k, r in enumerate(group):
                (answer,) = self._run_paillier(name, [r], slot)
                deliver(k, answer)
                answers.append(answer)
            return answers
        return self._run_paillier(name, group, slot)

    def _run_paillier(self, name: str, group: list[Request], slot: int) -> list[PaillierAnswer]:
        torch = self._torch
        p = self._paillier[name]
        stream = self._streams[slot]
        ctx = p["contexts"][slot]
        total = sum(r.queries for r in group)
        C, V, K = p["chunks"], p["vectors"], p["words"]
        dev = f"cuda:{self.device}"
        with torch.cuda.stream(stream):
            q = torch.cat([r.payload.to(dev, non_blocking=True) for r in group], dim=0)  # [B, C, K]
            qc = q.permute(1, 0, 2).contiguous()                                      # [C, B, K]
            out = torch.empty((C, total, V, K), dtype=torch.int32, device=dev)
            for c in range(C):
                ctx.mulmod_outer_array(qc[c], total, p["index"][c], V, out[c])
            done = torch.cuda.Event()
            done.record(stream)
        done.synchronize()
        # the merged launch wrote one buffer: its bytes return to the budget
        # when the last answer sharing it is released
        pending = [len(group)]
        lock = threading.Lock()
        group_bytes = sum(r.nbytes for r in group)

        def release_one() -> None:
            with lock:
                pending[0] -= 1
                last = pending[0] == 0
            if last:
                self.scheduler.release(group_bytes)

        answers, b0 = [], 0
        for r in group:
            answers.append(PaillierAnswer(out[:, b0:b0 + r.queries], release_one))
            b0 += r.queries
        return answers

    # -- the comparison point ------------------------------------------------
    def run_plain(self, kind: str, name: str, payload) -> Any:
        """One request alone: one launch per query, each waited for (no
        merging, no overlap).  Same answers as the served path."""
        torch = self._torch
        if kind == "bfv":
            from cuhepy_b200.bfv import _bfv_rns

            b = self._bfv[name]
            return _bfv_rns.search_index(b["server"], b["index"], payload, b["count"], b["compact"])
        p = self._paillier[name]
        ctx = p["contexts"][0]
        stream = self._streams[0]
        C, V, K = p["chunks"], p["vectors"], p["words"]
        dev = f"cuda:{self.device}"
        q = torch.as_tensor(payload)
        if q.dtype != torch.int32:
            q = q.view(torch.int32) if q.dtype == torch.uint32 else q.to(torch.int32)
        if q.dim() == 2:
            q = q.unsqueeze(1)
        with torch.cuda.stream(stream):
            q = q.to(dev)
            out = torch.empty((C, q.shape[0], V, K), dtype=torch.int32, device=dev)
        for b in range(int(q.shape[0])):
            for c in range(C):
                ctx.mulmod_outer_array(q[b, c].contiguous(), 1, p["index"][c], V, out[c, b])
                stream.synchronize()
        return out
