"""The allocation-free counting entry point, evx_count_static.

It exists for callers that cannot call cudaMalloc when they run a query: a
process whose device memory is entirely reserved by another allocator (a
framework's caching allocator, a serving process that pre-reserves its
budget), or code that must keep working when no device memory is left.  Its
only scratch is a fixed device array inside the library.  This file runs last
so that, if it fails, a run that stops at the first failure has already run
every other test; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from everest_b200 import capi, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

QUERIES = [
    ([0, 1, 2], [1, 2, 0], 4000),        # triangle: last edge closes on root nodes
    ([0, 0, 0], [1, 2, 1], 4000),        # last edge closes on the root pair (range arithmetic)
    ([0, 0, 0], [1, 2, 2], 4000),        # last edge closes on the new node (scan)
    ([0, 1, 1], [1, 2, 3], 2500),        # last edge maps a new node
    ([0, 1], [1, 0], 6000),              # two edges
    ([0, 1, 2, 3], [1, 2, 3, 0], 3000),  # four-edge cycle
    ([0, 1, 2, 3, 1], [1, 2, 3, 1, 4], 2000),
]


SPEC = synth.GraphSpec("static-zipf", "zipf", 800, 30_000, seed=17, t_max=300_000)


@pytest.fixture(scope="module")
def edges():
    return synth.generate(SPEC)


@pytest.fixture(scope="module")
def graph(edges):
    u, v, t = edges
    dg = capi.DeviceGraph(capi.graph_build_host(u, v, t), 0)
    yield dg
    dg.free()


def _worker_counts(graph, beg=0, end=-1):
    w = capi.Worker(0)
    want = []
    for mu, mv, d in QUERIES:
        w.take(graph, mu, mv, d, beg, end)
        want.append(w.run())
    w.close()
    return want


def test_static_count_equals_worker_and_oracle_twice(graph, edges):
    want = _worker_counts(graph)
    assert sum(want) > 0
    g = O.Graph(*edges, SPEC.num_nodes)
    assert want == [O.count(g, mu, mv, d)[0] for mu, mv, d in QUERIES]
    first = capi.count_static(graph, QUERIES)
    second = capi.count_static(graph, QUERIES)  # the array keeps the last call's contents
    assert first == want
    assert second == want
    # a single query reusing slot 0 after a larger call
    assert capi.count_static(graph, QUERIES[3:4]) == want[3:4]


def test_static_count_root_window_on_a_worker_stream(graph, edges):
    beg, end = 4_000, 21_000
    want = _worker_counts(graph, beg, end)
    g = O.Graph(*edges, SPEC.num_nodes)
    assert want == [O.count(g, mu, mv, d, roots=(beg, end))[0] for mu, mv, d in QUERIES]
    side = capi.Worker(0)  # owns a non-default stream
    try:
        for _ in range(2):
            assert capi.count_static(graph, QUERIES, beg, end, stream=side.stream) == want
    finally:
        side.close()


def test_static_count_bad_last_query_launches_nothing(graph):
    want = _worker_counts(graph)
    bad = QUERIES + [([0, 1, 2], [1, 2, 0], -5)]  # negative delta: rejected
    with pytest.raises(capi.EvxError):
        capi.count_static(graph, bad)
    assert capi.count_static(graph, QUERIES) == want


def test_static_count_rejects_too_many_queries(graph):
    qs = [QUERIES[0]] * (capi.STATIC_MAX_QUERIES + 1)
    with pytest.raises(capi.EvxError) as ei:
        capi.count_static(graph, qs)
    assert ei.value.code == -1
    assert "256" in str(ei.value)
