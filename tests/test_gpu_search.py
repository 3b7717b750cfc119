"""Parity of the sm_100a search kernels (through the C ABI) with the oracle
and with the golden fixtures produced by the reference's own Baseline code."""
import json
import os

import numpy as np
import pytest

from everest_b200 import capi, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "golden.json")
SMALL = os.path.join(HERE, "golden", "small_graphs.npz")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def small_graphs():
    z = np.load(SMALL)
    names = sorted({k.rsplit("_", 1)[0] for k in z.files})
    return {n: (z[f"{n}_u"], z[f"{n}_v"], z[f"{n}_t"], int(z[f"{n}_V"][0])) for n in names}


@pytest.fixture(scope="module")
def worker():
    w = capi.Worker(0)
    yield w
    w.close()


def device_graph(u, v, t, ids=None):
    host = capi.graph_build_host(u, v, t, ids)
    return capi.DeviceGraph(host, 0)


def gpu_count(worker, dg, mu, mv, delta, beg=0, end=-1, flags=0):
    worker.take(dg, mu, mv, delta, beg, end, 0, flags)
    return worker.run()


def test_golden_small_graph_counts(golden, small_graphs, worker):
    by_graph = {}
    for c in golden["cases"]:
        by_graph.setdefault(c["graph"], []).append(c)
    n = 0
    for gname, cases in by_graph.items():
        u, v, t, V = small_graphs[gname]
        dg = device_graph(u, v, t)
        for c in cases:
            rb, re_ = c.get("roots", [0, -1])
            got = gpu_count(worker, dg, c["mu"], c["mv"], c["delta"], rb, re_)
            assert got == c["count"], (gname, c["motif"], c["delta"], got, c["count"])
            if n % 5 == 0:  # the directory-counted last level on a subset
                got3 = gpu_count(worker, dg, c["mu"], c["mv"], c["delta"], rb, re_,
                                 flags=capi.FLAG_PAIR_DIR)
                assert got3 == c["count"], (gname, c["motif"], c["delta"], got3, "pair dir")
            if n % 4 == 1:  # without the closing-endpoint check on a subset
                got5 = gpu_count(worker, dg, c["mu"], c["mv"], c["delta"], rb, re_,
                                 flags=capi.FLAG_NO_CLOSING_PRUNE)
                assert got5 == c["count"], (gname, c["motif"], c["delta"], got5, "no prune")
            if n % 3 == 0:  # the scanned closing edge on a subset
                got4 = gpu_count(worker, dg, c["mu"], c["mv"], c["delta"], rb, re_,
                                 flags=capi.FLAG_CLOSING_SCAN)
                assert got4 == c["count"], (gname, c["motif"], c["delta"], got4, "closing scan")
            if n % 6 == 2:  # mid-level closing edges scanned in the shorter list on a subset
                got6 = gpu_count(worker, dg, c["mu"], c["mv"], c["delta"], rb, re_,
                                 flags=capi.FLAG_LIST_SCAN)
                assert got6 == c["count"], (gname, c["motif"], c["delta"], got6, "list scan")
            if n % 8 == 3:  # without the per-root window bound on a subset
                got7 = gpu_count(worker, dg, c["mu"], c["mv"], c["delta"], rb, re_,
                                 flags=capi.FLAG_NO_ROOT_BOUND)
                assert got7 == c["count"], (gname, c["motif"], c["delta"], got7, "no root bound")
            if n % 7 == 0:  # the scanning last level on a subset
                got2 = gpu_count(worker, dg, c["mu"], c["mv"], c["delta"], rb, re_,
                                 flags=capi.FLAG_NO_PAIR_INDEX)
                assert got2 == c["count"], (gname, c["motif"], c["delta"], got2, "no pair index")
            if c["reference_baseline"] is not None:
                assert got == c["reference_baseline"]
            n += 1
        dg.free()
    assert n > 1000


def test_golden_zipf_200k(golden, worker):
    full = golden["full_zipf"]
    spec = synth.SPECS[full["graph"]]
    u, v, t = synth.generate(spec)
    import hashlib
    h = hashlib.sha256()
    for a in (u, v, t):
        h.update(np.ascontiguousarray(a, np.int32).tobytes())
    assert h.hexdigest() == full["digest"], "generator output drifted"
    dg = device_graph(u, v, t)
    tri = full["triangle"]
    assert gpu_count(worker, dg, tri["mu"], tri["mv"], tri["delta"]) == tri["count"]
    assert tri["count"] == tri["reference_baseline"]
    assert gpu_count(worker, dg, tri["mu"], tri["mv"], tri["delta"],
                     flags=capi.FLAG_STRICT_TS) == tri["strict_ts_count"]
    for p in full["patterns"]:
        assert gpu_count(worker, dg, p["mu"], p["mv"], p["delta"]) == p["count"], p["motif"]
        assert gpu_count(worker, dg, p["mu"], p["mv"], p["delta"],
                         flags=capi.FLAG_NO_PAIR_INDEX) == p["count"], p["motif"]
        assert gpu_count(worker, dg, p["mu"], p["mv"], p["delta"],
                         flags=capi.FLAG_PAIR_DIR) == p["count"], p["motif"]
        assert gpu_count(worker, dg, p["mu"], p["mv"], p["delta"],
                         flags=capi.FLAG_CLOSING_SCAN) == p["count"], p["motif"]
        assert gpu_count(worker, dg, p["mu"], p["mv"], p["delta"],
                         flags=capi.FLAG_STRICT_TS | capi.FLAG_CLOSING_SCAN) == gpu_count(
            worker, dg, p["mu"], p["mv"], p["delta"],
            flags=capi.FLAG_STRICT_TS | capi.FLAG_NO_PAIR_INDEX), p["motif"]
        assert gpu_count(worker, dg, p["mu"], p["mv"], p["delta"],
                         flags=capi.FLAG_STRICT_TS) == gpu_count(
            worker, dg, p["mu"], p["mv"], p["delta"],
            flags=capi.FLAG_STRICT_TS | capi.FLAG_NO_PAIR_INDEX), p["motif"]
    dg.free()


def test_random_tiny_vs_brute_force(worker):
    rng = np.random.default_rng(123)
    for trial in range(150):
        E = int(rng.integers(0, 28))
        V = int(rng.integers(2, 6))
        u = rng.integers(0, V, E).astype(np.int32)
        v = rng.integers(0, V, E).astype(np.int32)
        t = np.sort(rng.integers(0, 15, E)).astype(np.int32)
        k = int(rng.integers(2, 6))
        pat = synth.random_patterns(1, (k, k), (2, min(k + 1, 5)), seed=trial)[0]
        mu = [a for a, b in pat]
        mv = [b for a, b in pat]
        delta = int(rng.integers(0, 10))
        want = len(O.brute_force(u, v, t, mu, mv, delta))
        dg = device_graph(u, v, t)
        for flags in (0, capi.FLAG_NO_STEAL, capi.FLAG_NO_PAIR_INDEX, capi.FLAG_PAIR_DIR, capi.FLAG_CLOSING_SCAN,
                      capi.FLAG_NO_CLOSING_PRUNE, capi.FLAG_NO_CLOSING_PRUNE | capi.FLAG_NO_PAIR_INDEX,
                      capi.FLAG_LIST_SCAN, capi.FLAG_LIST_SCAN | capi.FLAG_NO_STEAL, capi.FLAG_NO_ROOT_BOUND,
                      capi.FLAG_NO_ROOT_BOUND | capi.FLAG_NO_PAIR_INDEX,
                      capi.FLAG_NO_ROOT_BOUND | capi.FLAG_NO_CLOSING_PRUNE, capi.FLAG_NO_ROOT_BOUND | capi.FLAG_NEW_SCAN,
                      capi.FLAG_NO_ROOT_BOUND | capi.FLAG_PAIR_DIR):
            assert gpu_count(worker, dg, mu, mv, delta, flags=flags) == want, (trial, pat, delta, flags)
        strict = len(O.brute_force(u, v, t, mu, mv, delta, strict_ts=True))
        assert gpu_count(worker, dg, mu, mv, delta, flags=capi.FLAG_STRICT_TS) == strict
        assert gpu_count(worker, dg, mu, mv, delta, flags=capi.FLAG_STRICT_TS | capi.FLAG_CLOSING_SCAN) == strict
        assert gpu_count(worker, dg, mu, mv, delta, flags=capi.FLAG_STRICT_TS | capi.FLAG_LIST_SCAN) == strict
        assert gpu_count(worker, dg, mu, mv, delta, flags=capi.FLAG_STRICT_TS | capi.FLAG_NO_ROOT_BOUND) == strict
        dg.free()


def test_tuning_variants_agree(small_graphs, worker):
    u, v, t, V = small_graphs["mid-hub"]
    g = O.Graph(u, v, t, V)
    dg = device_graph(u, v, t)
    pats = [([0, 1, 2], [1, 2, 0]), ([0, 0, 0], [1, 2, 1]), ([0, 1, 2, 3], [1, 2, 3, 0]),
            ([0, 1, 2, 3, 1], [1, 2, 3, 1, 4])]
    try:
        for mu, mv in pats:
            want, _ = O.count(g, mu, mv, 2000)
            for tun in [(256, 0, 32, 16, 2), (32, 1, 1, 1, 2), (128, 2, 7, 0, 2),
                        (64, 0, 64, 4, 8), (256, 1, 1024, 2, 2)]:
                worker.set_tuning(*tun)
                assert gpu_count(worker, dg, mu, mv, 2000) == want, (mu, mv, tun)
    finally:
        worker.set_tuning()
        dg.free()


def test_root_ranges(small_graphs, worker):
    u, v, t, V = small_graphs["mid-uniform"]
    g = O.Graph(u, v, t, V)
    dg = device_graph(u, v, t)
    mu, mv = [0, 1, 2], [1, 2, 0]
    total = 0
    bounds = [0, 1, 17, 500, 1234, g.E - 2]
    for a, b in zip(bounds[:-1], bounds[1:]):
        want, _ = O.count(g, mu, mv, 400, roots=(a, b))
        got = gpu_count(worker, dg, mu, mv, 400, a, b)
        assert got == want
        total += got
    assert total == O.count(g, mu, mv, 400)[0]
    assert gpu_count(worker, dg, mu, mv, 400, 5, 5) == 0
    dg.free()


def test_edge_cases(worker):
    # empty graph, fewer edges than motif edges, all self-loops
    dg = device_graph(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert gpu_count(worker, dg, [0, 1, 2], [1, 2, 0], 10) == 0
    dg.free()
    dg = device_graph(np.array([0, 1], np.int32), np.array([1, 2], np.int32),
                      np.array([1, 2], np.int32))
    assert gpu_count(worker, dg, [0, 1, 2], [1, 2, 0], 10) == 0
    assert gpu_count(worker, dg, [0, 1], [1, 2], 10) == 1
    dg.free()
    dg = device_graph(np.array([3, 3, 3], np.int32), np.array([3, 3, 3], np.int32),
                      np.array([1, 1, 1], np.int32))
    assert gpu_count(worker, dg, [0, 0], [1, 1], 10) == 0
    dg.free()


def test_overflow_rejected(worker):
    big = np.iinfo(np.int32).max - 5
    dg = device_graph(np.array([0, 1], np.int32), np.array([1, 0], np.int32),
                      np.array([big - 1, big], np.int32))
    with pytest.raises(capi.EvxError) as ei:
        worker.take(dg, [0, 1], [1, 0], 100)
    assert ei.value.code == -4
    worker.take(dg, [0, 1], [1, 0], 5)
    assert worker.run() == 1
    dg.free()


def test_bad_motif_rejected(worker):
    dg = device_graph(np.array([0], np.int32), np.array([1], np.int32), np.array([1], np.int32))
    for mu, mv in (([0, 2], [1, 3]), ([0, 1], [1, 1]), ([1, 0], [0, 2])):
        with pytest.raises(capi.EvxError):
            worker.take(dg, mu, mv, 1)
    with pytest.raises(capi.EvxError):
        worker.take(dg, [0] * 9, list(range(1, 10)), 1)
    dg.free()


def test_enumeration_golden_rows(golden, small_graphs, worker):
    for c in golden["enum_cases"]:
        u, v, t, V = small_graphs[c["graph"]]
        ids = np.arange(u.size, dtype=np.int32)[::-1].copy()  # distinct original line ids
        dg = device_graph(u, v, t, ids)
        cap = c["total"] + 5
        worker.take(dg, c["mu"], c["mv"], c["delta"], 0, -1, cap)
        cnt = worker.run()
        assert cnt == c["total"]
        rows = worker.enum_rows(cap)
        want = sorted(ids[np.array(r, dtype=np.int64)].tolist() for r in c["rows"])
        got = sorted(rows.tolist())
        assert got == want
        dg.free()


def test_enumeration_cap_rule(small_graphs, worker):
    """count > cap: exactly cap rows, each a valid match, no duplicates; with
    EXACT_TOTAL the count is the exact total."""
    u, v, t, V = small_graphs["mid-ties"]
    g = O.Graph(u, v, t, V)
    mu, mv = [0, 1, 2, 3], [1, 2, 3, 0]
    delta = 10
    rows_all, total = O.enumerate_rows(g, mu, mv, delta, 10 ** 7)
    assert total > 50
    valid = set(map(tuple, rows_all.tolist()))
    dg = device_graph(u, v, t)
    cap = total // 3
    worker.take(dg, mu, mv, delta, 0, -1, cap)
    cnt = worker.run()
    assert cnt >= cap
    rows = worker.enum_rows(cap)
    assert rows.shape == (cap, 4)
    got = list(map(tuple, rows.tolist()))
    assert len(set(got)) == cap
    assert set(got) <= valid
    worker.take(dg, mu, mv, delta, 0, -1, cap, capi.FLAG_EXACT_TOTAL)
    assert worker.run() == total
    dg.free()


def test_enumeration_random_tiny_vs_brute_force(worker):
    """Enumerated rows equal brute force's on random tiny graphs, for motifs
    whose middle edges join mapped nodes (pair-run walks) and otherwise, with
    the pair-run walk on and off."""
    rng = np.random.default_rng(321)
    pats = [([0, 1, 0], [1, 0, 1]), ([0, 0, 1], [1, 1, 0]), ([0, 1, 1, 2], [1, 2, 0, 0]),
            ([0, 1, 2, 1], [1, 2, 0, 2]), ([0, 1, 2, 3], [1, 2, 3, 0]), ([0, 1, 1, 0], [1, 0, 0, 1])]
    for trial in range(60):
        E = int(rng.integers(0, 30))
        V = int(rng.integers(2, 6))
        u = rng.integers(0, V, E).astype(np.int32)
        v = rng.integers(0, V, E).astype(np.int32)
        t = np.sort(rng.integers(0, 12, E)).astype(np.int32)
        mu, mv = pats[trial % len(pats)]
        delta = int(rng.integers(0, 9))
        want = sorted(map(tuple, O.brute_force(u, v, t, mu, mv, delta)))
        dg = device_graph(u, v, t)
        for flags in (0, capi.FLAG_LIST_SCAN, capi.FLAG_NO_STEAL, capi.FLAG_NO_ROOT_BOUND):
            worker.take(dg, mu, mv, delta, 0, -1, len(want) + 4, flags)
            assert worker.run() == len(want), (trial, mu, mv, delta, flags)
            got = sorted(map(tuple, worker.enum_rows(len(want) + 4).tolist()))
            assert got == want, (trial, mu, mv, delta, flags)
        dg.free()


def test_enumeration_matches_count_zipf(worker):
    spec = synth.SPECS["zipf-10k-200k"]
    u, v, t = synth.generate(spec)
    g = O.Graph(u, v, t, spec.num_nodes)
    dg = device_graph(u, v, t)
    mu, mv = [0, 1, 2], [1, 2, 0]
    want, _ = O.count(g, mu, mv, 600)
    rows_o, tot = O.enumerate_rows(g, mu, mv, 600, want + 1)
    worker.take(dg, mu, mv, 600, 0, -1, want + 10)
    assert worker.run() == want
    rows = worker.enum_rows(want + 10)
    assert sorted(map(tuple, rows.tolist())) == sorted(map(tuple, rows_o.tolist()))
    dg.free()
