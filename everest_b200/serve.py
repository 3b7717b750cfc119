"""Serving loop: continuous batching of motif queries on resident graphs.

The reference answers one query at a time and re-uploads the graph for each
(system/tmine/frontend.py:69-96, system/batch-query.py:14-20).  Here:

* graphs stay resident on the device (``add_graph``);
* ``submit`` returns a future immediately; a loop thread admits requests:
  - count queries are packed into batches (one persistent launch each, see
    ``capi.Batch``); up to ``inflight_batches`` batches run at once on their
    own streams, so requests that arrive while others are on the GPU are
    admitted as soon as a batch slot frees up;
  - enumerate queries run as single-query searches on their own streams,
    admitted only when the device has room for their row buffers
    (cap x k x 4 bytes plus a reserve) and an enumeration slot is free;
* completed work is detected without blocking (CUDA event queries), futures
  are resolved and each request's latency (submit -> result) is recorded;
* an optional work limit keeps heavy queries out of the shared batches
  (work = adjacency records examined inside their time windows, fixed by
  the graph and the query): a query past it is stopped on the device and
  re-queued for the heavy slots: workers that run it with no limit, one
  root range (chunk) at a time -- each chunk launched on a fraction of the
  SMs (heavy_blocks_per_sm) while other work is queued or running and on
  the whole GPU otherwise, so that it overlaps the batches instead of
  holding them back, and several slots share one heavy query's chunks.  Its result (the sum over its chunks; an
  enumeration or a constrained query runs as one chunk) is exact like
  every other (``Result.requeued`` says it took that route).  With
  ``heavy_slots=0`` a query past the limit is resolved with
  ``Result.limited`` set and no count instead.

Results are independent of the mix: every query keeps its own counters in
the batch (one per query) or its own worker.
"""
from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import capi


@dataclass
class Request:
    graph: str
    mu: Sequence[int]
    mv: Sequence[int]
    delta: int
    enum_cap: int = 0
    flags: int = 0
    beg: int = 0          # root edge ids [beg, end); end < 0 = to the last root
    end: int = -1
    constraints: Optional[object] = None  # compiled everest_b200.constraints.Constraints
    submitted: float = field(default_factory=time.perf_counter)
    future: Future = field(default_factory=Future)


@dataclass
class HeavyJob:
    """A query re-run on the heavy slots, root range by root range."""
    req: Request
    next_root: int
    end_root: int
    chunk: int
    acc: int = 0
    inflight: int = 0
    rows: Optional[np.ndarray] = None


@dataclass
class Result:
    count: Optional[int]
    rows: Optional[np.ndarray] = None
    latency_s: float = 0.0
    limited: bool = False   # stopped at the work limit and not re-run (count is None)
    requeued: bool = False  # passed the work limit and was re-run on a heavy slot


class Server:
    def __init__(self, device: int = 0, max_batch: int = 64, inflight_batches: int = 2,
                 enum_slots: int = 2, mem_reserve: int = 1 << 30, idle_sleep_s: float = 50e-6,
                 backend=None, limit: int = 0, use_graph: bool = False, tile_roots: int = 64,
                 enum_blocks_per_sm: int = 2, batch_share: float = 1.0, heavy_slots: int = 2,
                 heavy_blocks_per_sm: int = 2, heavy_chunks: int = 64):
        # backend: the module providing Batch, Worker, DeviceGraph and
        # device_mem_info (the C-ABI binding; tests substitute a fake)
        self.be = backend if backend is not None else capi
        capi_ = self.be
        self.device = device
        self.max_batch = max_batch
        self.mem_reserve = mem_reserve
        self.idle_sleep_s = idle_sleep_s
        self.graphs: Dict[str, capi.DeviceGraph] = {}
        self.count_q: "collections.deque[Request]" = collections.deque()
        self.enum_q: "collections.deque[Request]" = collections.deque()
        self.lock = threading.Lock()
        self.cv = threading.Condition(self.lock)
        self.limit = int(limit)
        self.tile_roots = int(tile_roots)
        self.use_graph = bool(use_graph)
        # fraction of a batch kernel's usual resident blocks per SM: below 1,
        # two batches in flight run side by side instead of the second one
        # waiting for the first one's blocks
        self.batch_share = float(batch_share)
        self.batches = [capi_.Batch(device, max_batch) for _ in range(inflight_batches)]
        for b in self.batches:
            if self.limit:
                b.set_limit(self.limit)
            # served batches change shape from one launch to the next, so a
            # captured CUDA graph would be re-instantiated almost every time:
            # launch directly unless asked otherwise.  Small tiles: one heavy
            # query of a batch then spreads over many warps instead of
            # holding the whole batch back on a few
            if hasattr(b, "set_tuning"):
                b.set_tuning(tile_roots=tile_roots, use_graph=use_graph)
        self.batch_reqs: List[Optional[List[Request]]] = [None] * inflight_batches
        self.enum_workers = [capi_.Worker(device) for _ in range(enum_slots)]
        for w in self.enum_workers:
            if self.limit:
                w.set_limit(self.limit)
        # an enumeration's kernel holds its blocks until it ends: while count
        # work is queued or running, run it on a fraction of the SMs
        # (blocks_per_sm of the usual 4-8) so that count batches still find
        # room; with no count work about, on the whole GPU
        self.enum_blocks_per_sm = int(enum_blocks_per_sm)
        self.enum_reqs: List[Optional[Request]] = [None] * enum_slots
        # heavy slots: queries that passed the work limit, re-run without it
        self.heavy_q: "collections.deque[HeavyJob]" = collections.deque()
        self.heavy_workers = [capi_.Worker(device) for _ in range(heavy_slots if self.limit else 0)]
        # per slot: (job, first root, end root) of the chunk it runs
        self.heavy_reqs: List[Optional[tuple]] = [None] * len(self.heavy_workers)
        self.heavy_chunks = max(1, int(heavy_chunks))
        self.heavy_t0: List[float] = [0.0] * len(self.heavy_workers)
        self.heavy_blocks_per_sm = int(heavy_blocks_per_sm)
        self.requeued = 0
        self.latencies: List[float] = []
        # (kind, launch time, completion time, queries) of every launch
        self.launch_log: List[tuple] = []
        self.batch_t0: List[float] = [0.0] * inflight_batches
        self.enum_t0: List[float] = [0.0] * enum_slots
        self.completed = 0
        self.limited = 0
        self.batches_launched = 0
        self.first_submit: Optional[float] = None
        self.last_done: Optional[float] = None
        self.error: Optional[BaseException] = None
        self.running = True
        self.thread = threading.Thread(target=self._loop, name="evx-serve", daemon=True)
        self.thread.start()

    # ------------------------------------------------------------- API --
    def add_graph(self, name: str, host: capi.HostGraph, node_features=None, edge_features=None) -> None:
        """Make a graph resident; node features (per relabeled vertex) and
        edge features (per sorted edge) serve constrained queries."""
        g = self.be.DeviceGraph(host, self.device)
        if node_features is not None or edge_features is not None:
            g.set_features(node_features, edge_features)
        self.graphs[name] = g

    def submit(self, graph: str, mu, mv, delta: int, enum_cap: int = 0, flags: int = 0, beg: int = 0,
               end: int = -1, constraints=None) -> Future:
        """Queue a query; roots are the edge ids [beg, end) (the whole graph
        by default), as in the reference's MineJob(data, delta, beg, end).
        constraints: the YAML constraint keys (a dict) or a compiled
        everest_b200.constraints.Constraints; a constrained query runs on a
        worker slot, like an enumeration."""
        if graph not in self.graphs:
            raise KeyError(f"graph {graph!r} is not resident")
        if isinstance(constraints, dict):
            from .constraints import Constraints
            constraints = Constraints.from_yaml(constraints, list(mu), list(mv))
        if constraints is not None and constraints.empty:
            constraints = None
        r = Request(graph, list(mu), list(mv), int(delta), int(enum_cap), int(flags), int(beg), int(end),
                    constraints)
        with self.cv:
            if self.first_submit is None:
                self.first_submit = r.submitted
            (self.enum_q if (enum_cap > 0 or constraints is not None) else self.count_q).append(r)
            self.cv.notify()
        return r.future

    def stats(self) -> dict:
        lat = np.array(self.latencies) if self.latencies else np.zeros(1)
        span = (self.last_done - self.first_submit) if (self.last_done and self.first_submit) else 0.0
        return {"completed": self.completed, "limited": self.limited, "requeued": self.requeued,
                "batches": self.batches_launched,
                "queries_per_s": self.completed / span if span > 0 else 0.0,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "p999_ms": float(np.percentile(lat, 99.9) * 1e3), "max_ms": float(lat.max() * 1e3),
                "longest_launches_ms": sorted(([k, round((t1 - t0) * 1e3, 2), n] for k, t0, t1, n in self.launch_log),
                                              key=lambda x: -x[1])[:5]}

    def drain(self, timeout_s: float = 600.0) -> None:
        t0 = time.time()
        while True:
            with self.lock:
                busy = self._busy()
            if not busy:
                return
            if self.error:
                raise self.error
            if time.time() - t0 > timeout_s:
                raise TimeoutError("serving queue did not drain")
            time.sleep(0.001)

    def close(self) -> None:
        with self.cv:
            self.running = False
            self.cv.notify()
        self.thread.join(timeout=60)
        for b in self.batches:
            b.close()
        for w in self.enum_workers + self.heavy_workers:
            w.close()
        for g in self.graphs.values():
            if hasattr(g, "free"):
                g.free()
        self.graphs.clear()

    # ------------------------------------------------------------ loop --
    def _busy(self) -> bool:
        return bool(self.count_q or self.enum_q or self.heavy_q or any(self.batch_reqs) or any(self.enum_reqs)
                    or any(self.heavy_reqs))

    def _requeue(self, reqs: List[Request]) -> None:
        """Queries past the work limit: run them again on the heavy slots
        (the caller holds the lock).  A count query is cut into about
        heavy_chunks root ranges; an enumeration (its cap spans every root)
        or a constrained query runs as one."""
        self.requeued += len(reqs)
        for r in reqs:
            g = self.graphs[r.graph]
            E = getattr(g, "num_edges", None)
            beg = max(0, r.beg)
            if E is None:
                end = r.end
                chunk = 0  # unknown graph size: one chunk, the request's own range
            else:
                top = max(0, int(E) - len(r.mu) + 1)
                end = top if r.end < 0 else min(r.end, int(E))
                if end <= beg:  # no roots: nothing to re-run
                    self._finish(r, Result(0, np.zeros((0, len(r.mu)), np.int32) if r.enum_cap > 0 else None,
                                           requeued=True))
                    continue
                one = r.enum_cap > 0 or r.constraints is not None
                chunk = (end - beg) if one else -(-(end - beg) // self.heavy_chunks)
            self.heavy_q.append(HeavyJob(r, beg, end, chunk))

    def _finish(self, r: Request, res: Result) -> None:
        now = time.perf_counter()
        res.latency_s = now - r.submitted
        self.latencies.append(res.latency_s)
        self.completed += 1
        self.limited += 1 if res.limited else 0
        self.last_done = now
        r.future.set_result(res)

    def _poll(self) -> bool:
        progressed = False
        for i, b in enumerate(self.batches):
            reqs = self.batch_reqs[i]
            if reqs is not None and b.done():
                self.launch_log.append(("batch", self.batch_t0[i], time.perf_counter(), len(reqs)))
                counts = b.result()
                b.clear()
                again = [r for r, c in zip(reqs, counts) if c == capi.LIMITED] if self.heavy_workers else []
                with self.lock:  # re-queued and released together: drain() always sees them
                    self._requeue(again)
                    self.batch_reqs[i] = None
                for r, c in zip(reqs, counts):
                    lim = c == capi.LIMITED
                    if not (lim and self.heavy_workers):
                        self._finish(r, Result(None if lim else c, limited=lim))
                progressed = True
        for i, w in enumerate(self.enum_workers):
            r = self.enum_reqs[i]
            if r is not None and w.done():
                kind = "enumerate" if r.enum_cap > 0 else "constrained"
                self.launch_log.append((kind, self.enum_t0[i], time.perf_counter(), 1))
                try:
                    c, lim = w.result(), False
                except capi.LimitExceeded:
                    c, lim = None, True
                with self.lock:
                    self._requeue([r] if (lim and self.heavy_workers) else [])
                    self.enum_reqs[i] = None
                if not (lim and self.heavy_workers):
                    rows = w.enum_rows(r.enum_cap) if r.enum_cap > 0 else None
                    self._finish(r, Result(c, rows, limited=lim))
                progressed = True
        for i, w in enumerate(self.heavy_workers):
            slot = self.heavy_reqs[i]
            if slot is not None and w.done():
                job = slot[0]
                r = job.req
                self.launch_log.append(("heavy", self.heavy_t0[i], time.perf_counter(), 1))
                job.acc += w.result()
                if r.enum_cap > 0:
                    job.rows = w.enum_rows(r.enum_cap)
                with self.lock:
                    job.inflight -= 1
                    done = job.inflight == 0 and job.next_root >= job.end_root and \
                        (not self.heavy_q or self.heavy_q[0] is not job)
                    self.heavy_reqs[i] = None
                if done:
                    self._finish(r, Result(job.acc, job.rows, requeued=True))
                progressed = True
        return progressed

    def _admit(self) -> bool:
        progressed = False
        # count queries: fill free batch slots.  A batch holds one graph and
        # one motif size: the persistent kernel is instantiated for the
        # largest motif of its batch, and a smaller motif run in a larger
        # instantiation pays for its registers and shared memory.
        for i, b in enumerate(self.batches):
            if self.batch_reqs[i] is not None:
                continue
            with self.lock:
                if not self.count_q:
                    break
                key = (self.count_q[0].graph, len(self.count_q[0].mu))
                take = []
                rest = collections.deque()
                while self.count_q and len(take) < self.max_batch:
                    r = self.count_q.popleft()
                    (take if (r.graph, len(r.mu)) == key else rest).append(r)
                rest.extend(self.count_q)
                self.count_q = rest
                # claimed under the lock: drain() never sees the requests in
                # neither the queue nor a slot
                self.batch_reqs[i] = take
            for r in take:
                b.add(self.graphs[r.graph], r.mu, r.mv, r.delta, r.beg, r.end, r.flags)
            if self.batch_share < 1.0 and hasattr(b, "set_tuning"):
                full = 8 if key[1] <= 3 else (6 if key[1] == 4 else 4)  # the kernels' register budgets
                b.set_tuning(tile_roots=self.tile_roots, blocks_per_sm=max(1, int(full * self.batch_share)),
                             use_graph=self.use_graph)
            b.launch()
            self.batch_t0[i] = time.perf_counter()
            self.batches_launched += 1
            progressed = True
        # enumerate queries: admission by the memory their row buffers need
        for i, w in enumerate(self.enum_workers):
            if self.enum_reqs[i] is not None:
                continue
            with self.lock:
                if not self.enum_q:
                    break
                r = self.enum_q[0]
            need = r.enum_cap * len(r.mu) * 4
            free, _ = self.be.device_mem_info(self.device)
            if need + self.mem_reserve > free:
                break  # wait for running work to release memory
            with self.lock:
                self.enum_q.popleft()
                self.enum_reqs[i] = r  # claimed under the lock (see the batches above)
            if r.constraints is not None:
                w.take(self.graphs[r.graph], r.mu, r.mv, r.delta, r.beg, r.end, r.enum_cap, r.flags,
                       constraints=r.constraints)
            else:
                w.take(self.graphs[r.graph], r.mu, r.mv, r.delta, r.beg, r.end, r.enum_cap, r.flags)
            if self.enum_blocks_per_sm and hasattr(w, "set_tuning"):
                busy = bool(self.count_q) or any(x is not None for x in self.batch_reqs)
                w.set_tuning(block=128, blocks_per_sm=self.enum_blocks_per_sm if busy else 0, roots_per_fetch=32,
                             steal_interval=16, min_split=2)
            w.launch()
            self.enum_t0[i] = time.perf_counter()
            progressed = True
        # heavy queries: chunk by chunk, no work limit, on a fraction of the
        # SMs while other work is queued or running (the whole GPU otherwise)
        for i, w in enumerate(self.heavy_workers):
            if self.heavy_reqs[i] is not None:
                continue
            with self.lock:
                if not self.heavy_q:
                    break
                job = self.heavy_q[0]
                r = job.req
            if r.enum_cap > 0:
                need = r.enum_cap * len(r.mu) * 4
                free, _ = self.be.device_mem_info(self.device)
                if need + self.mem_reserve > free:
                    break
            with self.lock:
                if job.chunk <= 0:
                    b0, b1 = r.beg, r.end  # the request's own range, as submitted
                    job.next_root = job.end_root
                else:
                    b0 = job.next_root
                    b1 = min(job.end_root, b0 + job.chunk)
                    job.next_root = b1
                job.inflight += 1
                if job.next_root >= job.end_root:
                    self.heavy_q.popleft()  # every chunk handed out
                self.heavy_reqs[i] = (job, b0, b1)
            if r.constraints is not None:
                w.take(self.graphs[r.graph], r.mu, r.mv, r.delta, b0, b1, r.enum_cap, r.flags,
                       constraints=r.constraints)
            else:
                w.take(self.graphs[r.graph], r.mu, r.mv, r.delta, b0, b1, r.enum_cap, r.flags)
            if hasattr(w, "set_tuning"):
                # beside other work a heavy chunk takes a fraction of the SMs
                # (a persistent kernel holds its blocks until it ends); alone
                # it takes the whole GPU.  Capping it always was measured
                # worse: served p99 1.34x FIFO's against 0.68x.
                busy = bool(self.count_q or self.enum_q) or any(x is not None for x in self.batch_reqs) \
                    or any(x is not None for x in self.enum_reqs)
                w.set_tuning(block=128, blocks_per_sm=self.heavy_blocks_per_sm if busy else 0,
                             roots_per_fetch=32, steal_interval=16, min_split=2)
            w.launch()
            self.heavy_t0[i] = time.perf_counter()
            progressed = True
        return progressed

    def _loop(self) -> None:
        try:
            while True:
                with self.cv:
                    if not self.running:
                        return
                    idle = not self._busy()
                    if idle:
                        self.cv.wait(timeout=0.05)
                        continue
                p1 = self._poll()
                p2 = self._admit()
                if not (p1 or p2):
                    time.sleep(self.idle_sleep_s)
        except BaseException as e:  # surface loop failures to callers
            self.error = e
            with self.lock:
                pending = list(self.count_q) + list(self.enum_q)
                pending += [r for reqs in self.batch_reqs if reqs for r in reqs]
                pending += [r for r in self.enum_reqs if r]
                pending += [j.req for j in self.heavy_q] + [s[0].req for s in self.heavy_reqs if s]
            for r in pending:
                if not r.future.done():
                    r.future.set_exception(e)
