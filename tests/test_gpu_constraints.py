"""Constrained search on the GPU (through the C ABI) against the counts of
the reference's own generated search code (tests/golden/
constraint_golden.json) and the constrained oracle."""
import json
import os

import numpy as np
import pytest

from everest_b200 import capi, synth
from everest_b200.constraints import Constraints
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def worker():
    w = capi.Worker(0)
    yield w
    w.close()


def upload(u, v, t, nf=None, ef=None):
    """Device graph with features re-indexed to its relabeled vertices."""
    host = capi.graph_build_host(u, v, t)
    dg = capi.DeviceGraph(host, 0)
    if nf is not None or ef is not None:
        node = None
        if nf is not None:
            node = np.asarray(nf, np.int32)[host.original_vertex_ids(u, v)]
        dg.set_features(node, None if ef is None else np.asarray(ef, np.int32)[: host.num_edges])
    return dg


def run(worker, dg, mu, mv, delta, cons, enum_cap=0, flags=0, beg=0, end=-1):
    worker.take(dg, mu, mv, delta, beg, end, enum_cap, flags, constraints=cons)
    return worker.run()


def test_reference_generated_counts(worker):
    with open(os.path.join(GOLD, "constraint_golden.json")) as f:
        cases = json.load(f)["cases"]
    d = np.load(os.path.join(GOLD, "small_graphs.npz"))
    feats = np.load(os.path.join(GOLD, "constraint_features.npz"))
    by_graph = {}
    for c in cases:
        by_graph.setdefault(c["graph"], []).append(c)
    n = 0
    for gname, cs in by_graph.items():
        u, v, t = d[gname + "_u"], d[gname + "_v"], d[gname + "_t"]
        dg = upload(u, v, t, feats[gname + "_node"], feats[gname + "_edge"])
        for c in cs:
            cons = Constraints.from_yaml(c["constraints"], c["mu"], c["mv"])
            got = run(worker, dg, c["mu"], c["mv"], c["delta"], cons)
            assert got == c["count"], (gname, c["motif"], c["constraints"], got, c["count"])
            # both searches give the same counts: node / edge / gap-only
            # queries on the warp-synchronous one, every query on the per-lane one
            got2 = run(worker, dg, c["mu"], c["mv"], c["delta"], cons, flags=capi.FLAG_PER_LANE)
            assert got2 == c["count"], (gname, c["motif"], c["constraints"], got2, "per lane")
            if not cons.to_struct().anti_mask and not cons.to_struct().has_filter:
                got3 = run(worker, dg, c["mu"], c["mv"], c["delta"], cons, flags=capi.FLAG_WARP_SYNC)
                assert got3 == c["count"], (gname, c["motif"], c["constraints"], got3, "warp sync")
            n += 1
        dg.free()
    assert n == len(cases)


def _bursty(E, V, seed):
    return synth.generate(synth.GraphSpec(f"cons-{E}", "bursty", V, E, seed=seed, t_span=50 * E))


CONS = [
    ([0, 1, 2, 2, 3], [1, 2, 0, 3, 0], {"antiEdge": [False, False, True, False, False], "node": "f % 4 != 0",
                                         "temporal": [3000, 6000, 6000, 3000]}),
    ([0, 1, 2, 3], [1, 2, 3, 0], {"node0": "f > 3", "node1": "f < 8", "node2": "f > 1", "node3": "f != 5",
                                  "edge": "f % 5 != 2", "filter": "e0 + e1 + e2 + e3 > 12"}),
    ([0, 0, 0], [1, 2, 3], {"temporal": [2000, 500], "edge": "(f & 3) != 1"}),
    ([0, 1, 0], [1, 0, 1], {"filter": "e0 * e2 - e1 > 10"}),
    # warp-synchronous constrained search (no anti-edge, no filter)
    ([0, 1, 2, 3], [1, 2, 3, 0], {"node0": "f > 3", "node1": "f < 8", "node2": "f > 1", "node3": "f != 5"}),
    ([0, 1, 2, 3], [1, 2, 3, 0], {"node": "f % 3 != 0", "temporal": [4000, 8000, 3000]}),
    ([0, 1, 1, 0], [1, 0, 2, 2], {"edge": "f % 4 != 1", "node2": "f > 4", "node0": "f > 0", "node1": "f > 0"}),
    ([0, 0, 1, 2], [1, 2, 2, 0], {"temporal": [9000, 2000, 2000]}),
    ([0, 1, 2], [1, 0, 1], {"node": "f > 2"}),
]


def test_large_graph_against_oracle(worker):
    """A 400k-edge graph with hubs: every constraint kind at once, against
    the constrained oracle."""
    u, v, t = _bursty(400_000, 20_000, 11)
    rng = np.random.Generator(np.random.PCG64(12))
    nf = rng.integers(0, 10, 20_000).astype(np.int32)
    ef = rng.integers(0, 10, u.size).astype(np.int32)
    g = O.Graph(u, v, t, 20_000)
    dg = upload(u, v, t, nf, ef)
    delta = 20_000
    for mu, mv, c in CONS:
        cons = Constraints.from_yaml(dict(c, delta=delta), mu, mv)
        want = O.count_constrained(g, mu, mv, delta, cons.to_struct(), nf, ef)
        got = run(worker, dg, mu, mv, delta, cons)
        assert got == want, (mu, mv, c, got, want)
        if "antiEdge" not in c and "filter" not in c:
            assert run(worker, dg, mu, mv, delta, cons, flags=capi.FLAG_WARP_SYNC) == want, (mu, mv, c)
        # a sub-range of roots
        want = O.count_constrained(g, mu, mv, delta, cons.to_struct(), nf, ef, roots=(1000, 90_000))
        assert run(worker, dg, mu, mv, delta, cons, beg=1000, end=90_000) == want
    dg.free()


def test_no_constraints_equals_plain_search(worker):
    u, v, t = _bursty(200_000, 10_000, 21)
    dg = upload(u, v, t)
    for mu, mv in (([0, 1, 2], [1, 2, 0]), ([0, 1, 2, 3], [1, 2, 3, 0]), ([0, 0, 1], [1, 2, 0])):
        empty = Constraints.from_yaml({"delta": 5000}, mu, mv)
        worker.take(dg, mu, mv, 5000)
        plain = worker.run()
        assert run(worker, dg, mu, mv, 5000, empty) == plain
    dg.free()


def test_enumeration_rows(worker):
    u, v, t = _bursty(100_000, 5_000, 31)
    rng = np.random.Generator(np.random.PCG64(32))
    nf = rng.integers(0, 10, 5_000).astype(np.int32)
    ef = rng.integers(0, 10, u.size).astype(np.int32)
    g = O.Graph(u, v, t, 5_000)
    dg = upload(u, v, t, nf, ef)
    mu, mv = [0, 1, 2], [1, 2, 0]
    cons = Constraints.from_yaml({"delta": 30_000, "node": "f > 2", "filter": "e0 + e2 > 6",
                                  "temporal": [20_000, 20_000]}, mu, mv)
    rows_o, total = O.enumerate_constrained(g, mu, mv, 30_000, cons.to_struct(), 10**6, nf, ef)
    assert 0 < total < 10**6
    got = run(worker, dg, mu, mv, 30_000, cons, enum_cap=total + 10)
    assert got == total
    rows = worker.enum_rows(total + 10)
    assert rows.shape == (total, 3)
    assert sorted(map(tuple, rows.tolist())) == sorted(map(tuple, rows_o.tolist()))
    # capped: exactly cap distinct valid rows; the exact total on request
    cap = max(1, total // 3)
    run(worker, dg, mu, mv, 30_000, cons, enum_cap=cap)
    part = worker.enum_rows(cap)
    assert part.shape == (cap, 3)
    keep = set(map(tuple, rows_o.tolist()))
    assert len(set(map(tuple, part.tolist()))) == cap and all(tuple(r) in keep for r in part.tolist())
    assert run(worker, dg, mu, mv, 30_000, cons, enum_cap=cap, flags=capi.FLAG_EXACT_TOTAL) == total
    dg.free()


def test_enumeration_rows_warp_synchronous(worker):
    """Node / edge predicates and temporal gaps without anti-edges or a
    filter: rows equal the oracle's on both searches (default routing, the
    per-lane search, the warp-synchronous search)."""
    u, v, t = _bursty(100_000, 5_000, 33)
    rng = np.random.Generator(np.random.PCG64(34))
    nf = rng.integers(0, 10, 5_000).astype(np.int32)
    ef = rng.integers(0, 10, u.size).astype(np.int32)
    g = O.Graph(u, v, t, 5_000)
    dg = upload(u, v, t, nf, ef)
    for mu, mv, c in (([0, 1, 2], [1, 2, 0], {"node": "f > 2", "temporal": [20_000, 20_000]}),
                      ([0, 1, 2, 0], [1, 0, 0, 2], {"edge": "f != 3", "node2": "f < 7", "node0": "f > 0",
                                                    "node1": "f > 0"})):
        cons = Constraints.from_yaml(dict(c, delta=30_000), mu, mv)
        rows_o, total = O.enumerate_constrained(g, mu, mv, 30_000, cons.to_struct(), 10**6, nf, ef)
        assert 0 < total < 10**6
        for flags in (0, capi.FLAG_PER_LANE, capi.FLAG_WARP_SYNC):
            assert run(worker, dg, mu, mv, 30_000, cons, enum_cap=total + 10, flags=flags) == total
            rows = worker.enum_rows(total + 10)
            assert sorted(map(tuple, rows.tolist())) == sorted(map(tuple, rows_o.tolist())), (mu, mv, c, flags)
    dg.free()


def test_checks(worker):
    u, v, t = _bursty(10_000, 500, 41)
    dg = upload(u, v, t)
    m4a = ([0, 1, 2, 2, 3], [1, 2, 0, 3, 0])
    good = Constraints.from_yaml({"delta": 100, "antiEdge": [False, False, True, False, False]}, *m4a)
    st = good.to_struct()
    st.anti_mask = 2  # motif edge 1
    with pytest.raises(capi.EvxError, match="cannot be anti-edges"):
        run(worker, dg, *m4a, 100, st)
    st.anti_mask = 4
    with pytest.raises(capi.EvxError, match="enumeration with anti-edges"):
        run(worker, dg, *m4a, 100, st, enum_cap=10)
    needs_nodes = Constraints.from_yaml({"delta": 100, "node": "f > 1"}, *m4a)
    with pytest.raises(capi.EvxError, match="node features"):
        run(worker, dg, *m4a, 100, needs_nodes)
    bad = good.to_struct()
    bad.has_filter = 1
    bad.filter.len = 2
    bad.filter.op[0], bad.filter.op[1] = 2, 6  # push a variable, then add: stack underflow
    dg.set_features(np.zeros(dg.num_vertices, np.int32), np.zeros(dg.num_edges, np.int32))
    with pytest.raises(capi.EvxError, match="stack underflow"):
        run(worker, dg, *m4a, 100, bad)
    # the worker still runs a plain job afterwards
    worker.take(dg, [0, 1, 2], [1, 2, 0], 100)
    worker.run()
    dg.free()
