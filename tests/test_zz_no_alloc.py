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


@pytest.fixture(scope="module")
def graph():
    spec = synth.GraphSpec("static-zipf", "zipf", 800, 30_000, seed=17, t_max=300_000)
    u, v, t = synth.generate(spec)
    dg = capi.DeviceGraph(capi.graph_build_host(u, v, t), 0)
    yield dg
    dg.free()


def test_static_count_equals_worker_twice(graph):
    w = capi.Worker(0)
    want = []
    for mu, mv, d in QUERIES:
        w.take(graph, mu, mv, d)
        want.append(w.run())
    w.close()
    assert sum(want) > 0
    first = capi.count_static(graph, QUERIES)
    second = capi.count_static(graph, QUERIES)  # the array keeps the last call's contents
    assert first == want
    assert second == want
    # a single query reusing slot 0 after a larger call
    assert capi.count_static(graph, QUERIES[3:4]) == want[3:4]


def test_static_count_rejects_too_many_queries(graph):
    qs = [QUERIES[0]] * (capi.STATIC_MAX_QUERIES + 1)
    with pytest.raises(capi.EvxError) as ei:
        capi.count_static(graph, qs)
    assert ei.value.code == -1
    assert "256" in str(ei.value)
