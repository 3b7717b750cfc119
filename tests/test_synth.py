"""Seeded synthetic workloads."""
import numpy as np

from everest_b200 import synth, workloads
from oracle import oracle as O


def test_three_edge_patterns_by_rule():
    pats = synth.three_edge_patterns()
    assert len(pats) == 36 and len({tuple(p) for p in pats}) == 36
    for p in pats:
        mu, mv = [a for a, b in p], [b for a, b in p]
        g = O.Graph(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32), 1)
        assert O.count(g, mu, mv, 1)[0] == 0  # accepted by the motif rules
        assert max(max(mu), max(mv)) <= 2


def test_random_patterns_rules():
    pats = synth.random_patterns(64, (3, 4), (2, 4), seed=3)
    assert len(pats) == 64 and len({tuple(p) for p in pats}) == 64
    for p in pats:
        assert p[0] == (0, 1) and 3 <= len(p) <= 4
        nn = 2
        for a, b in p[1:]:
            assert a != b and (a < nn or b < nn)
            nn = max(nn, a + 1, b + 1)
        assert 2 <= nn <= 4


def test_generators_sorted_and_deterministic():
    spec = synth.GraphSpec("t-bursty", "bursty", 5000, 40_000, seed=4)
    u, v, t = synth.generate(spec)
    u2, v2, t2 = synth.generate(spec)
    assert np.array_equal(u, u2) and np.array_equal(t, t2)
    assert u.size == 40_000 and np.all(np.diff(t) >= 0) and np.all(u != v)
    assert u.dtype == np.int32 and t.dtype == np.int32
    spec = synth.GraphSpec("t-zipf", "zipf", 100, 3000, seed=4)
    u, v, t = synth.generate(spec)
    assert np.all(u != v) and np.all(np.diff(t) >= 0) and t.max() < spec.t_max


def test_workload_queries():
    qs = workloads.queries("bursty-7.8m-3edge")
    assert len(qs) == 36 and all(q["delta"] == 86400 for q in qs)
    assert workloads.queries("zipf-200k-triangle")[0]["mu"] == [0, 1, 2]
