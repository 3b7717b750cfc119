"""Serving-loop admission logic on CPU with a fake device backend (the
oracle computes the counts; the backend only models slots, completion and
free memory)."""
import threading
import time

import numpy as np
import pytest

from everest_b200 import capi, serve, synth
from oracle import oracle as O


class FakeBackend:
    """Batch / Worker / DeviceGraph / device_mem_info with host semantics."""

    def __init__(self, graphs, free_bytes):
        self.graphs = graphs          # name -> oracle Graph
        self.free = free_bytes
        self.lock = threading.Lock()
        self.max_concurrent_enum = 0
        self.running_enum = 0
        self.enum_bps = []  # blocks per SM asked for at each enumeration launch
        self.batch_s = 0.002  # how long a launched batch takes
        self.features = {}    # name -> (node features, edge features)
        self.constrained = 0  # constrained launches

    def device_mem_info(self, device):
        with self.lock:
            return self.free, 1 << 40

    def DeviceGraph(self, host, device):
        return host  # the test passes the graph name as "host"

    def Batch(self, device, max_q):
        be = self

        class B:
            def __init__(self):
                self.q = []
                self.t_done = None
                self.limit = 0

            def set_limit(self, n):
                self.limit = n

            def add(self, g, mu, mv, d, beg, end, flags):
                self.q.append((g, mu, mv, d, beg, end))

            def launch(self):
                self.res = []
                for g, mu, mv, d, beg, end in self.q:
                    gr = be.graphs[g]
                    hi = O.default_roots(gr, len(mu))[1] if end < 0 else min(end, O.default_roots(gr, len(mu))[1])
                    c = O.count(gr, mu, mv, d, roots=(beg, max(beg, hi)))[0]
                    # the fake's work measure is the count itself
                    self.res.append(capi.LIMITED if self.limit and c > self.limit else c)
                self.t_done = time.perf_counter() + be.batch_s

            def done(self):
                return time.perf_counter() >= self.t_done

            def result(self):
                return self.res

            def clear(self):
                self.q = []

            def close(self):
                pass
        return B()

    def Worker(self, device):
        be = self

        class W:
            def set_limit(self, n):
                self.limit = n

            def set_tuning(self, block, blocks_per_sm, roots_per_fetch, steal_interval, min_split):
                be.enum_bps.append(blocks_per_sm)

            def take(self, g, mu, mv, d, beg, end, cap, flags, constraints=None):
                self.args = (g, mu, mv, d, cap)
                self.roots = (beg, end)
                self.cons = constraints

            def launch(self):
                g, mu, mv, d, cap = self.args
                with be.lock:
                    be.free -= cap * len(mu) * 4
                    be.running_enum += 1
                    be.max_concurrent_enum = max(be.max_concurrent_enum, be.running_enum)
                if self.cons is not None:
                    nf, ef = be.features[g]
                    be.constrained += 1
                    self.total = O.count_constrained(be.graphs[g], mu, mv, d, self.cons.to_struct(), nf, ef)
                    self.rows = None
                else:
                    gr = be.graphs[g]
                    beg, end = self.roots
                    top = O.default_roots(gr, len(mu))[1]
                    hi = top if end < 0 else min(end, top)
                    roots = (beg, max(beg, hi))
                    if cap > 0:
                        self.rows, self.total = O.enumerate_rows(gr, mu, mv, d, cap, roots=roots)
                    else:
                        self.rows, self.total = None, O.count(gr, mu, mv, d, roots=roots)[0]
                self.t_done = time.perf_counter() + 0.003

            def done(self):
                return time.perf_counter() >= self.t_done

            def result(self):
                g, mu, mv, d, cap = self.args
                with be.lock:
                    be.free += cap * len(mu) * 4
                    be.running_enum -= 1
                return min(self.total, self.total)

            def enum_rows(self, n):
                return self.rows[:n]

            def close(self):
                pass
        return W()


@pytest.fixture(scope="module")
def graph():
    spec = synth.GraphSpec("serve-zipf", "zipf", 200, 3000, seed=6, t_max=30_000)
    u, v, t = synth.generate(spec)
    return O.Graph(u, v, t, spec.num_nodes)


def test_results_same_alone_and_in_mix(graph):
    be = FakeBackend({"g": graph}, free_bytes=1 << 40)
    srv = serve.Server(max_batch=8, inflight_batches=2, enum_slots=2, mem_reserve=0, backend=be)
    srv.add_graph("g", "g")
    qs = [([0, 1, 2], [1, 2, 0], 2000), ([0, 0, 0], [1, 2, 1], 3000), ([0, 1], [1, 0], 4000),
          ([0, 1, 2, 3], [1, 2, 3, 0], 3000)] * 6
    futs = [srv.submit("g", mu, mv, d) for mu, mv, d in qs]
    efut = srv.submit("g", [0, 1, 2], [1, 2, 0], 2000, enum_cap=50)
    srv.drain(60)
    for (mu, mv, d), f in zip(qs, futs):
        assert f.result(1).count == O.count(graph, mu, mv, d)[0]
    er = efut.result(1)
    assert er.rows.shape[0] == min(50, O.count(graph, [0, 1, 2], [1, 2, 0], 2000)[0])
    st = srv.stats()
    assert st["completed"] == len(qs) + 1 and st["batches"] >= len(qs) // 8
    assert st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    srv.close()


def test_enumeration_admission_waits_for_memory(graph):
    # room for one enumeration buffer at a time
    cap = 1000
    be = FakeBackend({"g": graph}, free_bytes=cap * 3 * 4 + 100)
    srv = serve.Server(max_batch=4, inflight_batches=1, enum_slots=3, mem_reserve=50, backend=be)
    srv.add_graph("g", "g")
    futs = [srv.submit("g", [0, 1, 2], [1, 2, 0], 1000 + 500 * i, enum_cap=cap) for i in range(5)]
    srv.drain(60)
    assert all(f.result(1).count >= 0 for f in futs)
    assert be.max_concurrent_enum == 1
    srv.close()


def test_unknown_graph_rejected(graph):
    be = FakeBackend({"g": graph}, free_bytes=1 << 40)
    srv = serve.Server(backend=be)
    with pytest.raises(KeyError):
        srv.submit("nope", [0, 1], [1, 0], 5)
    srv.close()


def test_root_ranges_and_count_limit(graph):
    # windows of roots, and a limit that stops the largest queries: those
    # come back flagged, every other count is exact
    be = FakeBackend({"g": graph}, free_bytes=1 << 40)
    E = graph.u.size
    qs = [([0, 1, 2], [1, 2, 0], 3000, 0, E // 2), ([0, 0, 0], [1, 2, 1], 3000, E // 3, E),
          ([0, 1], [1, 0], 4000, 100, 900), ([0, 0], [1, 1], 30_000, 0, -1)]
    exact = []
    for mu, mv, d, beg, end in qs:
        hi = O.default_roots(graph, len(mu))[1] if end < 0 else min(end, O.default_roots(graph, len(mu))[1])
        exact.append(O.count(graph, mu, mv, d, roots=(beg, hi))[0])
    limit = sorted(exact)[-2]  # the largest query passes it, the others do not
    # without heavy slots a query past the limit comes back flagged, with no count
    srv = serve.Server(max_batch=4, inflight_batches=1, enum_slots=1, mem_reserve=0, backend=be, limit=limit,
                       heavy_slots=0)
    srv.add_graph("g", "g")
    futs = [srv.submit("g", mu, mv, d, beg=beg, end=end) for mu, mv, d, beg, end in qs]
    srv.drain(60)
    for f, c in zip(futs, exact):
        r = f.result(1)
        if c > limit:
            assert r.limited and r.count is None
        else:
            assert not r.limited and r.count == c
    assert srv.stats()["limited"] == sum(c > limit for c in exact) == 1
    srv.close()
    # with heavy slots (the default) it is re-run without the limit: every
    # query gets its exact count
    srv = serve.Server(max_batch=4, inflight_batches=1, enum_slots=1, mem_reserve=0, backend=be, limit=limit)
    srv.add_graph("g", "g")
    futs = [srv.submit("g", mu, mv, d, beg=beg, end=end) for mu, mv, d, beg, end in qs]
    srv.drain(60)
    for f, c in zip(futs, exact):
        r = f.result(1)
        assert not r.limited and r.count == c
        assert r.requeued == (c > limit)
    st = srv.stats()
    assert st["limited"] == 0 and st["requeued"] == 1 and st["completed"] == len(qs)
    assert any(k == "heavy" for k, *_ in srv.launch_log)
    srv.close()


class _SizedName(str):
    """A graph handle of the fake backend that knows its edge count (the
    server cuts heavy queries into root ranges with it)."""


def test_heavy_query_runs_in_root_chunks(graph):
    be = FakeBackend({"g": graph}, free_bytes=1 << 40)
    sized = _SizedName("g")
    sized.num_edges = graph.u.size
    be.DeviceGraph = lambda host, device: sized
    mu, mv, d = [0, 1, 2], [1, 2, 0], 3000
    exact = O.count(graph, mu, mv, d)[0]
    small = O.count(graph, [0, 1], [1, 0], 400)[0]
    srv = serve.Server(max_batch=4, inflight_batches=1, enum_slots=1, mem_reserve=0, backend=be,
                       limit=max(small, 1), heavy_slots=2, heavy_chunks=5)
    srv.add_graph("g", "g")
    f_heavy = srv.submit("g", mu, mv, d)
    f_small = srv.submit("g", [0, 1], [1, 0], 400)
    srv.drain(60)
    r = f_heavy.result(1)
    assert r.requeued and not r.limited and r.count == exact
    assert f_small.result(1).count == small and not f_small.result(1).requeued
    assert sum(1 for k, *_ in srv.launch_log if k == "heavy") == 5  # five root ranges
    assert srv.stats()["requeued"] == 1
    srv.close()


def test_enumerations_share_the_gpu_only_beside_count_work(graph):
    # enumerations launched while count queries are queued or running take
    # the configured fraction of the SMs; alone they take the whole GPU (0)
    be = FakeBackend({"g": graph}, free_bytes=1 << 40)
    be.batch_s = 0.2  # count batches still running when the first enumeration arrives
    srv = serve.Server(max_batch=4, inflight_batches=1, enum_slots=1, mem_reserve=0, backend=be,
                       enum_blocks_per_sm=2)
    srv.add_graph("g", "g")
    futs = [srv.submit("g", [0, 1, 2], [1, 2, 0], 2000) for _ in range(12)]
    futs.append(srv.submit("g", [0, 1, 2], [1, 2, 0], 2000, enum_cap=10))
    srv.drain(60)
    futs.append(srv.submit("g", [0, 1, 2], [1, 2, 0], 2000, enum_cap=10))
    srv.drain(60)
    assert all(f.result(1) is not None for f in futs)
    assert be.enum_bps[0] == 2 and be.enum_bps[-1] == 0
    srv.close()


def test_constrained_queries_run_on_worker_slots(graph):
    be = FakeBackend({"g": graph}, free_bytes=1 << 40)
    rng = np.random.Generator(np.random.PCG64(3))
    be.features["g"] = (rng.integers(0, 10, graph.V).astype(np.int32),
                        rng.integers(0, 10, graph.E).astype(np.int32))
    srv = serve.Server(max_batch=8, inflight_batches=2, enum_slots=2, mem_reserve=0, backend=be)
    srv.add_graph("g", "g")
    cons = [({"node": "f > 3"}, [0, 1, 2], [1, 2, 0], 3000),
            ({"temporal": [800, 400], "edge": "f % 3 != 0"}, [0, 0, 0], [1, 2, 3], 2000),
            ({"antiEdge": [False, False, True, False], "filter": "e0 + e3 > 8"}, [0, 1, 1, 2], [1, 2, 0, 0], 4000),
            ({}, [0, 1], [1, 0], 4000)]  # no constraint: a plain batched count
    futs = [srv.submit("g", mu, mv, d, constraints=c) for c, mu, mv, d in cons]
    plain = srv.submit("g", [0, 1, 2], [1, 2, 0], 3000)
    srv.drain(60)
    from everest_b200.constraints import Constraints
    nf, ef = be.features["g"]
    for (c, mu, mv, d), f in zip(cons, futs):
        want = O.count_constrained(graph, mu, mv, d, Constraints.from_yaml(c, mu, mv).to_struct(), nf, ef)
        res = f.result(1)
        assert res.count == want and res.rows is None
    assert plain.result(1).count == O.count(graph, [0, 1, 2], [1, 2, 0], 3000)[0]
    assert be.constrained == 3  # the empty set went to a batch
    assert any(k == "constrained" for k, *_ in srv.launch_log)
    srv.close()
