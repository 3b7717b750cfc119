"""Batched queries in one persistent launch (CUDA-graph replay) against
per-query launches and the oracle: every result is the same alone and in
the mix."""
import numpy as np
import pytest

from everest_b200 import capi, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    spec = synth.GraphSpec("batch-bursty", "bursty", 20_000, 150_000, seed=31, t_span=3_000_000)
    u, v, t = synth.generate(spec)
    dg = capi.DeviceGraph(capi.graph_build_host(u, v, t), 0)
    g = O.Graph(u, v, t, spec.num_nodes)
    yield dg, g
    dg.free()


def mixed_queries():
    qs = []
    for i, p in enumerate(synth.three_edge_patterns()):
        qs.append(([a for a, b in p], [b for a, b in p], [600, 3600, 20000][i % 3]))
    for i, p in enumerate(synth.random_patterns(16, (2, 5), (2, 4), seed=77)):
        qs.append(([a for a, b in p], [b for a, b in p], [900, 5000][i % 2]))
    return qs


def test_batch_equals_single_and_oracle(setup):
    dg, g = setup
    qs = mixed_queries()
    w = capi.Worker(0)
    single = []
    for mu, mv, d in qs:
        w.take(dg, mu, mv, d)
        single.append(w.run())
    w.close()
    for (mu, mv, d), c in list(zip(qs, single))[::5]:
        assert c == O.count(g, mu, mv, d)[0]
    b = capi.Batch(0, 256)
    for mu, mv, d in qs:
        b.add(dg, mu, mv, d)
    first = b.run()
    second = b.run()  # replay of the captured graph
    assert first == single and second == single
    b.set_tuning(tile_roots=64, use_graph=False)
    assert b.run() == single
    b.set_tuning(tile_roots=1024, steal_interval=0)
    assert b.run() == single
    b.close()


def test_batch_recomposition_and_single(setup):
    dg, g = setup
    qs = mixed_queries()
    b = capi.Batch(0, 64)
    for mu, mv, d in qs[:10]:
        b.add(dg, mu, mv, d)
    r1 = b.run()
    b.clear()
    for mu, mv, d in qs[10:13]:
        b.add(dg, mu, mv, d)
    r2 = b.run()
    b.clear()
    mu, mv, d = qs[40]
    b.add(dg, mu, mv, d)
    r3 = b.run()
    b.clear()
    mu2, mv2, d2 = qs[7]
    b.add(dg, mu2, mv2, d2)  # same shape as the previous single-query batch: graph replay
    r4 = b.run()
    assert r1 == [O.count(g, m, n, x)[0] for m, n, x in qs[:10]]
    assert r2 == [O.count(g, m, n, x)[0] for m, n, x in qs[10:13]]
    assert r3 == [O.count(g, mu, mv, d)[0]]
    assert r4 == [O.count(g, mu2, mv2, d2)[0]]
    b.close()


def test_batch_root_ranges_and_errors(setup):
    dg, g = setup
    b = capi.Batch(0, 4)
    mu, mv = [0, 1, 2], [1, 2, 0]
    b.add(dg, mu, mv, 5000, 100, 40000)
    b.add(dg, mu, mv, 5000, 40000, -1)
    r = b.run()
    assert r[0] == O.count(g, mu, mv, 5000, roots=(100, 40000))[0]
    assert sum(r) == O.count(g, mu, mv, 5000, roots=(100, g.E - 2))[0]
    b.add(dg, mu, mv, 5000)
    b.add(dg, mu, mv, 5000)
    with pytest.raises(capi.EvxError):
        b.add(dg, mu, mv, 5000)  # full
    b.close()
