"""Autotuner: launch parameters per (motif, graph, delta) for count queries.

The reference fixes its launch shape (block 96, steal after 20 iterations,
host-driven tail expansion; system/templates/warpBalancing/top.snp:1,
system/templates/tailExpan/timeUp.snp:1-10).  Here the best setting depends
on the motif and the graph, so the tuner times a handful of candidates on a
root sample of the query (every candidate must return the same count on the
sample, which is checked) and caches the winner per key:

    key = (graph fingerprint, motif edges, floor(log2(delta + 1)))

Knobs: resident blocks per SM (0 = occupancy), intra-warp rebalance interval
and minimum split width ("steal granularity"), how the last edge is
counted: range arithmetic on the pair index, a pair hash-table or
pair-directory lookup per partial match, or a scan ("tail-expansion depth"),
whether an edge between two mapped nodes walks its pair run or scans the
shorter adjacency list, and whether each root's window is bounded by the
last edge's list.  Batches are tuned on
their tile size.
"""
from __future__ import annotations

import json
import math
import os
import threading
from typing import Dict, Optional, Sequence, Tuple

from . import capi

DEFAULT = {"blocks_per_sm": 0, "steal_interval": 16, "min_split": 2, "flags": 0}
CANDIDATES = [
    DEFAULT,
    {"blocks_per_sm": 0, "steal_interval": 4, "min_split": 2, "flags": 0},
    {"blocks_per_sm": 0, "steal_interval": 64, "min_split": 4, "flags": 0},
    {"blocks_per_sm": 0, "steal_interval": 0, "min_split": 2, "flags": capi.FLAG_NO_STEAL},
    {"blocks_per_sm": 0, "steal_interval": 16, "min_split": 2, "flags": capi.FLAG_NO_PAIR_INDEX},
    {"blocks_per_sm": 0, "steal_interval": 16, "min_split": 2, "flags": capi.FLAG_PAIR_DIR},
    {"blocks_per_sm": 0, "steal_interval": 4, "min_split": 2, "flags": capi.FLAG_PAIR_DIR},
    {"blocks_per_sm": 0, "steal_interval": 16, "min_split": 2, "flags": capi.FLAG_CLOSING_SCAN},
    {"blocks_per_sm": 0, "steal_interval": 4, "min_split": 2, "flags": capi.FLAG_CLOSING_SCAN},
    {"blocks_per_sm": 0, "steal_interval": 4, "min_split": 2, "flags": capi.FLAG_NO_CLOSING_PRUNE},
    {"blocks_per_sm": 0, "steal_interval": 4, "min_split": 2, "flags": capi.FLAG_NEW_SCAN},
    {"blocks_per_sm": 4, "steal_interval": 16, "min_split": 2, "flags": 0},
    {"blocks_per_sm": 0, "steal_interval": 16, "min_split": 2, "flags": capi.FLAG_LIST_SCAN},
    {"blocks_per_sm": 0, "steal_interval": 16, "min_split": 2, "flags": capi.FLAG_NO_ROOT_BOUND},
    {"blocks_per_sm": 0, "steal_interval": 4, "min_split": 2, "flags": capi.FLAG_NO_ROOT_BOUND},
    {"blocks_per_sm": 0, "steal_interval": 64, "min_split": 4, "flags": capi.FLAG_NO_ROOT_BOUND},
    {"blocks_per_sm": 0, "steal_interval": 4, "min_split": 2,
     "flags": capi.FLAG_NO_CLOSING_PRUNE | capi.FLAG_NO_ROOT_BOUND},
    {"blocks_per_sm": 0, "steal_interval": 4, "min_split": 2, "flags": capi.FLAG_NEW_SCAN | capi.FLAG_NO_ROOT_BOUND},
    {"blocks_per_sm": 0, "steal_interval": 16, "min_split": 2, "flags": capi.FLAG_PAIR_DIR | capi.FLAG_NO_ROOT_BOUND},
]
BATCH_TILES = (64, 128, 256, 512)


def graph_key(graph: capi.DeviceGraph) -> str:
    return f"{graph.name or 'graph'}:{graph.num_edges}:{graph.num_vertices}"


def query_key(graph: capi.DeviceGraph, mu: Sequence[int], mv: Sequence[int], delta: int) -> str:
    return f"{graph_key(graph)}|{','.join(map(str, mu))}|{','.join(map(str, mv))}|{int(math.log2(delta + 1))}"


class Autotuner:
    def __init__(self, device: int = 0, cache_path: Optional[str] = None, sample_roots: int = 400_000,
                 reps: int = 2):
        self.device = device
        self.cache_path = cache_path
        self.sample_roots = sample_roots
        self.reps = reps
        self.cache: Dict[str, dict] = {}
        self.lock = threading.Lock()
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.cache = json.load(f)

    def save(self) -> None:
        if self.cache_path:
            tmp = self.cache_path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)
            os.replace(tmp, self.cache_path)

    @staticmethod
    def apply(worker: capi.Worker, cfg: dict) -> int:
        """Set a worker's launch parameters; returns the flags to pass to take()."""
        worker.set_tuning(block=128, blocks_per_sm=cfg["blocks_per_sm"], roots_per_fetch=32,
                          steal_interval=cfg["steal_interval"], min_split=cfg["min_split"])
        return cfg["flags"]

    def tune(self, graph: capi.DeviceGraph, mu, mv, delta: int, worker: Optional[capi.Worker] = None) -> dict:
        key = query_key(graph, mu, mv, delta)
        with self.lock:
            if key in self.cache:
                return self.cache[key]
        own = worker is None
        w = worker or capi.Worker(self.device)
        E = graph.num_edges
        # a middle slice (away from the empty start of the time range), or
        # every root when sample_roots <= 0
        S = E if self.sample_roots <= 0 else min(E, self.sample_roots)
        beg = max(0, (E - S) // 2)
        best, best_ms, ref_count = None, float("inf"), None
        trials = []
        try:
            for cfg in CANDIDATES:
                flags = self.apply(w, cfg)
                times = []
                count = None
                for _ in range(self.reps):
                    w.take(graph, mu, mv, delta, beg, beg + S, 0, flags)
                    count = w.run()
                    times.append(w.last_stats()["device_ms"])
                if ref_count is None:
                    ref_count = count
                elif count != ref_count:
                    raise RuntimeError(f"autotune: candidate {cfg} changed the count ({count} != {ref_count})")
                ms = min(times)
                trials.append((cfg, ms))
                if ms < best_ms:
                    best, best_ms = cfg, ms
        finally:
            self.apply(w, DEFAULT)
            if own:
                w.close()
        entry = dict(best)
        entry["sample_ms"] = best_ms
        entry["default_ms"] = trials[0][1]
        with self.lock:
            self.cache[key] = entry
        return entry

    def count(self, graph: capi.DeviceGraph, mu, mv, delta: int, worker: capi.Worker) -> int:
        """Run a count query with its tuned parameters."""
        cfg = self.tune(graph, mu, mv, delta, worker)
        flags = self.apply(worker, cfg)
        worker.take(graph, mu, mv, delta, 0, -1, 0, flags)
        try:
            return worker.run()
        finally:
            self.apply(worker, DEFAULT)

    def tune_batch(self, batch_factory, queries, graph: capi.DeviceGraph, limit: int = 0) -> int:
        """Pick the tile size for a batch of (mu, mv, delta[, beg, end])
        queries; returns tile_roots (the batch's counts must not depend on
        it: checked; with a work limit the stopped queries must match too)."""
        best, best_ms, ref = BATCH_TILES[0], float("inf"), None
        for tr in BATCH_TILES:
            b = batch_factory()
            b.set_tuning(tile_roots=tr)
            if limit:
                b.set_limit(limit)
            for q in queries:
                b.add(graph, *q)
            r = b.run()
            r = b.run()
            ms = b.last_stats()["device_ms"]
            b.close()
            if ref is None:
                ref = r
            elif r != ref:
                raise RuntimeError("autotune: batch counts depend on the tile size")
            if ms < best_ms:
                best, best_ms = tr, ms
        return best
