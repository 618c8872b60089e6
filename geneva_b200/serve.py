"""Serving loop: continuous batching of matching requests plus mining jobs.

The reference serves nothing (one query per `gpumine` process).  Here a
server keeps one database resident and a batched session open (gva_session):

* matching requests (a .query text) are admitted between rounds, as long as
  their estimated frontier memory fits the admission budget, and join the
  running work at the next round; every round advances all admitted work one
  step, so a short query does not wait for a long one to finish;
* mining requests (max edges, min support) run on a worker thread with their
  own CUDA stream, so their rounds overlap the matching rounds on the device;
  they mine the graph database (graph support) or, when the server is given
  one data graph for mining, that graph (MNI support).  A mining run takes
  seconds, so at most `mine_queue_limit` of them wait behind the running one;
  a mining request arriving when that many wait is rejected at once
  (GenevaError, status REJECTED) instead of queueing without bound, which
  keeps the latency of every admitted mining request bounded by about
  (mine_queue_limit + 1) runs.

Latency of a request = completion time - arrival time (host wall clock).
"""
from __future__ import annotations

import ctypes
import os
import queue
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import Database, GenevaError, MODE_DV, Plan, _check, library, mine


REJECTED = 8  # status of a mining request refused by the admission policy (queue full)


@dataclass
class Request:
    kind: str                      # "match" | "mine"
    payload: object                # query text, or (max_edges, min_support)
    arrival: float = 0.0
    admitted: float = 0.0
    done: float = 0.0
    result: object = None
    future: Future = field(default_factory=Future)

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def _declare(lib):
    vp, u64, i32, u32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint32
    P = ctypes.POINTER
    lib.gva_session_create.argtypes = [vp, vp, u64, u32, P(vp)]
    lib.gva_session_create.restype = i32
    lib.gva_session_submit.argtypes = [vp, vp, P(u64), i32]
    lib.gva_session_submit.restype = i32
    lib.gva_session_round.argtypes = [vp, P(i32)]
    lib.gva_session_round.restype = i32
    lib.gva_session_poll.argtypes = [vp, P(u64), P(u64), P(u32), i32]
    lib.gva_session_poll.restype = i32
    lib.gva_session_free.argtypes = [vp]
    lib.gva_session_free.restype = None
    return lib


class Server:
    """One database, one open session, one mining worker."""

    def __init__(self, db: Database, budget_bytes: int = 150 << 30, support: bool = True,
                 slots: int = 4096, match_stream: Optional[int] = None, mine_stream: Optional[int] = None,
                 mine_db: Optional[Database] = None, mine_sm_percent: int = 50,
                 mine_host_threads: Optional[int] = None, mine_queue_limit: int = 2):
        """db: the graph database matching requests run against (and mining
        requests, with graph support, when mine_db is None).  mine_db: one
        data graph that mining requests run against with MNI support.
        Mining runs are long; they get at most mine_sm_percent of the SMs
        (MNI search kernel) and mine_host_threads host threads (default: half
        the cores), so that matching rounds keep GPU and host time.
        mine_queue_limit: mining requests that may wait behind the running
        one; later ones are rejected at arrival (status REJECTED)."""
        self.lib = _declare(library())
        self.db = db
        self._max_vertex_id = db.info()["max_vertex_id"]
        self.mine_db = mine_db
        self.mine_sm_percent = mine_sm_percent
        self.mine_host_threads = mine_host_threads if mine_host_threads is not None else max(1, (os.cpu_count() or 2) // 2)
        self.budget = budget_bytes
        self.support = support and db.num_graphs > 0
        self.mine_stream = mine_stream
        h = ctypes.c_void_p()
        _check(self.lib.gva_session_create(db._h, match_stream, budget_bytes, slots if self.support else 0,
                                           ctypes.byref(h)))
        self._ses = h
        self._slots = slots
        self._arrivals: "queue.Queue[Request]" = queue.Queue()
        self._mine_q: "queue.Queue[Optional[Request]]" = queue.Queue()
        self.mine_queue_limit = mine_queue_limit
        self.mine_rejected = 0
        self._waiting: List[Request] = []
        self._inflight = {}
        self._reserved = 0
        self._next_tag = 1
        self._stop = threading.Event()
        self._cancel = ctypes.c_int(0)  # set on close: a mining run in progress stops at its next round
        self.rounds = 0
        self.round_s: List[float] = []  # wall time of each round (host + device)
        self.completed: List[Request] = []
        self._lock = threading.Lock()
        self._loop = threading.Thread(target=self._run, daemon=True)
        self._miner = threading.Thread(target=self._run_mine, daemon=True)
        self._loop.start()
        self._miner.start()

    # ---- client side ------------------------------------------------------
    def submit_match(self, query_text: str) -> Request:
        r = Request("match", query_text, arrival=time.perf_counter())
        self._arrivals.put(r)
        return r

    def submit_mine(self, max_edges: int, min_support: int) -> Request:
        r = Request("mine", (max_edges, min_support), arrival=time.perf_counter())
        if self._mine_q.qsize() >= self.mine_queue_limit:
            r.done = r.arrival
            self.mine_rejected += 1
            r.future.set_exception(GenevaError(REJECTED, "mining queue full: request rejected at admission"))
            return r
        self._mine_q.put(r)
        return r

    def close(self):
        self._stop.set()
        # mining requests not started yet are cancelled; one in progress stops at its next round
        while True:
            try:
                r = self._mine_q.get_nowait()
            except queue.Empty:
                break
            if r is not None and not r.future.done():
                r.done = time.perf_counter()
                r.future.set_exception(GenevaError(5, "server closed before the request started"))
        self._cancel.value = 1
        self._mine_q.put(None)
        self._loop.join()
        self._miner.join()
        if self._ses:
            self.lib.gva_session_free(self._ses)
            self._ses = None

    # ---- admission --------------------------------------------------------
    def _estimate(self, plan: Plan, text: str) -> int:
        """Frontier bytes a request may pin: its widest rows over a seed-sized frontier."""
        k = max(2, text.count("\nv ") + (1 if text.startswith("v ") else 0))
        return 4 * k * (self._max_vertex_id // 4 + 1)

    def _admit(self):
        while True:
            try:
                self._waiting.append(self._arrivals.get_nowait())
            except queue.Empty:
                break
        wave, tags, plans = [], [], []
        keep = []
        for r in self._waiting:
            if len(self._inflight) + len(wave) >= self._slots:
                keep.append(r)
                continue
            try:
                plan = Plan.from_text(r.payload, MODE_DV)
            except GenevaError as e:
                r.done = time.perf_counter()
                r.result = e
                r.future.set_exception(e)
                continue
            est = self._estimate(plan, r.payload)
            if self._reserved + est > self.budget and self._inflight:
                keep.append(r)  # wait until memory frees up
                continue
            tag = self._next_tag
            self._next_tag += 1
            r.admitted = time.perf_counter()
            r._est = est
            r._plan = plan
            self._reserved += est
            self._inflight[tag] = r
            wave.append(r)
            tags.append(tag)
            plans.append(plan)
        self._waiting = keep
        if wave:
            arr = (ctypes.c_void_p * len(plans))(*[p._h.value for p in plans])
            t = (ctypes.c_uint64 * len(tags))(*tags)
            _check(self.lib.gva_session_submit(self._ses, arr, t, len(plans)))

    def _poll(self):
        cap = 256
        tags = (ctypes.c_uint64 * cap)()
        counts = (ctypes.c_uint64 * cap)()
        sups = (ctypes.c_uint32 * cap)()
        while True:
            n = self.lib.gva_session_poll(self._ses, tags, counts, sups, cap)
            if n < 0:
                raise GenevaError(3, self.lib.gva_last_error().decode())
            now = time.perf_counter()
            for i in range(n):
                r = self._inflight.pop(int(tags[i]))
                self._reserved -= r._est
                r.done = now
                r.result = (int(counts[i]), int(sups[i]) if self.support else None)
                r._plan.close()
                with self._lock:
                    self.completed.append(r)
                r.future.set_result(r.result)
            if n < cap:
                return

    def _run(self):
        active = ctypes.c_int(0)
        while True:
            self._admit()
            if self._inflight:
                t0 = time.perf_counter()
                st = self.lib.gva_session_round(self._ses, ctypes.byref(active))
                self.round_s.append(time.perf_counter() - t0)
                if st:
                    err = GenevaError(st, self.lib.gva_last_error().decode())
                    for r in self._inflight.values():
                        r.future.set_exception(err)
                    self._inflight.clear()
                    return
                self.rounds += 1
                self._poll()
            elif self._stop.is_set() and not self._waiting and self._arrivals.empty():
                return
            else:
                time.sleep(0.0002)

    def _run_mine(self):
        while True:
            r = self._mine_q.get()
            if r is None:
                return
            r.admitted = time.perf_counter()
            try:
                if self.mine_db is not None:
                    pats, stats = mine(self.mine_db, r.payload[0], r.payload[1], stream=self.mine_stream,
                                       support="mni", cancel=self._cancel, sm_percent=self.mine_sm_percent,
                                       host_threads=self.mine_host_threads)
                else:
                    pats, stats = mine(self.db, r.payload[0], r.payload[1], stream=self.mine_stream,
                                       cancel=self._cancel, host_threads=self.mine_host_threads)
                r.result = (pats, stats)
                r.done = time.perf_counter()
                with self._lock:
                    self.completed.append(r)
                r.future.set_result(r.result)
            except GenevaError as e:
                r.done = time.perf_counter()
                r.future.set_exception(e)


def percentile(xs, p):
    if not xs:
        return None
    return float(np.percentile(np.asarray(xs), p))
