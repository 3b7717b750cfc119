"""Work limits (evx_worker_set_limit / evx_batch_set_limit).  The work
measure (meter) is the number of adjacency records a query's search examines
inside their time windows; a query whose meter is at most the limit is
exact, a query above it is stopped early and flagged, alone and inside a
batch, and the boundary does not move between runs.  Capped enumeration
stops early too."""
import pytest

from everest_b200 import capi, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# out-star 0->1, 0->2, 0->3 on the 200k-edge Zipf graph: the top source
# sends ~38% of all edges, so a 50k-second window holds ~380 of its edges
# and the count is in the billions (about a second of search unlimited)
STAR = ([0, 0, 0], [1, 2, 3])
STAR_DELTA = 50_000


@pytest.fixture(scope="module")
def small():
    spec = synth.GraphSpec("limit-zipf", "zipf", 500, 20_000, seed=41, t_max=2_000_000)
    u, v, t = synth.generate(spec)
    dg = capi.DeviceGraph(capi.graph_build_host(u, v, t), 0)
    yield dg, O.Graph(u, v, t, spec.num_nodes)
    dg.free()


@pytest.fixture(scope="module")
def big():
    u, v, t = synth.load_or_generate("zipf-10k-200k")
    dg = capi.DeviceGraph(capi.graph_build_host(u, v, t), 0)
    yield dg
    dg.free()


QUERIES = [([0, 1, 2], [1, 2, 0], 50_000), ([0, 0, 0], [1, 2, 1], 20_000), ([0, 1], [1, 0], 100_000),
           ([0, 1, 2, 3], [1, 2, 3, 0], 40_000), ([0, 1, 1], [1, 2, 0], 30_000)]


def _run(w, dg, q, limit):
    w.set_limit(limit)
    w.take(dg, *q)
    try:
        return w.run(), False
    except capi.LimitExceeded as e:
        return e.count, True


def test_limit_boundary_is_exact_and_stable(small):
    dg, g = small
    w = capi.Worker(0)
    bisected = 0
    for q in QUERIES:
        c = O.count(g, *q)[0]
        assert c > 0
        assert _run(w, dg, q, 0) == (c, False)
        assert _run(w, dg, q, 1 << 40) == (c, False)
        if not _run(w, dg, q, 1)[1]:
            continue  # examines at most one record (e.g. a pair-index count)
        # bisect the smallest limit that lets the query finish
        lo, hi = 1, 1 << 40   # lo stops, hi finishes
        while hi - lo > 1:
            mid = (lo + hi) // 2
            cnt, lim = _run(w, dg, q, mid)
            if lim:
                lo = mid
            else:
                assert cnt == c
                hi = mid
        for _ in range(3):  # the boundary does not depend on scheduling
            assert _run(w, dg, q, hi) == (c, False)
            assert _run(w, dg, q, hi - 1)[1]
        bisected += 1
    assert bisected >= 3
    w.close()


def test_limit_stops_explosive_query_early(big):
    w = capi.Worker(0)
    total, lim = _run(w, big, (*STAR, STAR_DELTA), 0)
    t_full = w.last_stats()["device_ms"]
    assert not lim and total > 10**9
    cnt, lim = _run(w, big, (*STAR, STAR_DELTA), total // 1000)
    t_lim = w.last_stats()["device_ms"]
    assert lim and cnt < total
    assert t_lim < t_full / 5, (t_lim, t_full)
    w.close()


def test_batch_limit_flags_only_the_large_query(small, big):
    dg, g = small
    exact = [O.count(g, *q)[0] for q in QUERIES]
    # small-graph queries: the batch stops exactly the queries a worker
    # stops at the same limit, and every other count is exact
    w = capi.Worker(0)
    b = capi.Batch(0, 16)
    for q in QUERIES:
        b.add(dg, *q)
    for limit in (1, 300, 3000, 30_000, 10**12):
        alone = [_run(w, dg, q, limit) for q in QUERIES]
        b.set_limit(limit)
        for r in (b.run(), b.run()):  # launch and graph replay
            for (c, lim), x, ex in zip(alone, r, exact):
                assert (x == capi.LIMITED) == lim
                if not lim:
                    assert x == c == ex
    w.close()
    b.close()
    # big graph: the star is stopped; a cheap query beside it gets what it
    # gets alone under the same limit
    w = capi.Worker(0)
    star_total, _ = _run(w, big, (*STAR, STAR_DELTA), 0)
    lim = star_total // 100  # the star examines at least one record per match
    cheap = ([0, 1, 2], [1, 2, 0], 3600)
    cheap_alone = _run(w, big, cheap, lim)
    cheap_count, _ = _run(w, big, cheap, 0)
    w.close()
    b = capi.Batch(0, 16)
    b.set_limit(lim)
    b.add(big, *STAR, STAR_DELTA)
    b.add(big, *cheap)
    b.add(big, *STAR, STAR_DELTA, 1000, 150_000)
    r = b.run()
    assert r[0] == capi.LIMITED and r[2] == capi.LIMITED
    assert r[1] == (capi.LIMITED if cheap_alone[1] else cheap_alone[0])
    b.set_limit(0)
    r = b.run()
    assert r[0] == star_total and r[1] == cheap_count
    b.close()


def test_capped_enumeration_stops_early(big):
    # enumeration of the star with a small cap: rows are distinct valid
    # matches and the search ends long before the full count would
    w = capi.Worker(0)
    w.take(big, *STAR, STAR_DELTA)
    w.run()
    t_full = w.last_stats()["device_ms"]
    cap = 10_000
    w.take(big, *STAR, STAR_DELTA, 0, -1, cap)
    c = w.run()
    t_enum = w.last_stats()["device_ms"]
    rows = w.enum_rows(cap)
    assert c >= cap and rows.shape == (cap, 3)
    assert len({tuple(r) for r in rows.tolist()}) == cap
    assert t_enum < t_full / 5, (t_enum, t_full)
    w.close()
