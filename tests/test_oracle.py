"""The CPU oracle against the golden fixtures (produced by the host build of
the reference's own Baseline search body) and against brute force."""
import json
import os

import numpy as np
import pytest

from everest_b200 import synth
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(HERE, "golden", "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def small_graphs():
    z = np.load(os.path.join(HERE, "golden", "small_graphs.npz"))
    names = sorted({k.rsplit("_", 1)[0] for k in z.files})
    return {n: (z[f"{n}_u"], z[f"{n}_v"], z[f"{n}_t"], int(z[f"{n}_V"][0])) for n in names}


def test_golden_cases_pinned_by_reference(golden):
    cases = golden["cases"]
    assert len(cases) > 1000
    pinned = [c for c in cases if c["reference_baseline"] is not None]
    assert len(pinned) == len(cases)
    assert all(c["count"] == c["reference_baseline"] for c in pinned)


def test_oracle_reproduces_golden(golden, small_graphs):
    graphs = {n: O.Graph(u, v, t, V) for n, (u, v, t, V) in small_graphs.items()}
    for c in golden["cases"]:
        roots = tuple(c["roots"]) if "roots" in c else None
        got, _ = O.count(graphs[c["graph"]], c["mu"], c["mv"], c["delta"], roots=roots)
        assert got == c["count"], c


def test_reference_baseline_host_build_when_present(golden, small_graphs):
    if O.ref_lib() is None:
        pytest.skip("host build of the reference Baseline body not present")
    graphs = {n: O.Graph(u, v, t, V) for n, (u, v, t, V) in small_graphs.items()}
    for c in golden["cases"][::13]:
        roots = tuple(c["roots"]) if "roots" in c else None
        got = O.ref_baseline_count(graphs[c["graph"]], c["mu"], c["mv"], c["delta"], roots=roots,
                                   threads=2)
        assert got == c["count"], c


def test_full_zipf_triangle(golden):
    full = golden["full_zipf"]
    spec = synth.SPECS[full["graph"]]
    u, v, t = synth.generate(spec)
    g = O.Graph(u, v, t, spec.num_nodes)
    tri = full["triangle"]
    c, st = O.count(g, tri["mu"], tri["mv"], tri["delta"])
    assert c == tri["count"] == tri["reference_baseline"] == 221177
    assert st == tri["stats"]
    cs, _ = O.count(g, tri["mu"], tri["mv"], tri["delta"], strict_ts=True)
    assert cs == tri["strict_ts_count"]
    for p in full["patterns"][::5]:
        assert O.count(g, p["mu"], p["mv"], p["delta"])[0] == p["count"] == p["reference_baseline"]


def test_enumeration_golden(golden, small_graphs):
    for c in golden["enum_cases"]:
        u, v, t, V = small_graphs[c["graph"]]
        g = O.Graph(u, v, t, V)
        rows, tot = O.enumerate_rows(g, c["mu"], c["mv"], c["delta"], 10 ** 7)
        assert tot == c["total"] == len(c["rows"])
        assert sorted(rows.tolist()) == c["rows"]
        assert O.count(g, c["mu"], c["mv"], c["delta"])[0] == tot


def test_oracle_vs_brute_force():
    rng = np.random.default_rng(5)
    for trial in range(120):
        E = int(rng.integers(0, 24))
        V = int(rng.integers(2, 6))
        u = rng.integers(0, V, E).astype(np.int32)
        v = rng.integers(0, V, E).astype(np.int32)
        t = np.sort(rng.integers(0, 12, E)).astype(np.int32)
        k = int(rng.integers(2, 5))
        pat = synth.random_patterns(1, (k, k), (2, min(k + 1, 4)), seed=1000 + trial)[0]
        mu, mv = [a for a, b in pat], [b for a, b in pat]
        d = int(rng.integers(0, 8))
        g = O.Graph(u, v, t, V)
        bf = O.brute_force(u, v, t, mu, mv, d)
        assert O.count(g, mu, mv, d)[0] == len(bf)
        rows, tot = O.enumerate_rows(g, mu, mv, d, 10 ** 6)
        assert sorted(map(tuple, rows.tolist())) == bf
        assert O.count(g, mu, mv, d, strict_ts=True)[0] == len(O.brute_force(u, v, t, mu, mv, d, strict_ts=True))


def test_parse_reference_motifs(golden):
    txt = golden["reference_motifs"]
    assert set(txt) >= {f"M{i}" for i in range(1, 14)}
    assert O.parse_motif(txt["M2"]) == ([0, 0, 1], [1, 2, 3])
    assert O.parse_motif(txt["M4"]) == ([0, 1, 2, 3], [1, 2, 3, 0])
    assert O.parse_motif(txt["M3"]) == ([0, 1, 2, 3], [1, 2, 3, 1])
    for name, t in txt.items():
        mu, mv = O.parse_motif(t)
        nm = np.zeros(16, np.int32)
        assert O.lib().oracle_count is not None
        assert len(mu) == len(mv) >= 3


def test_bad_motif_rejected():
    g = O.Graph(np.array([0], np.int32), np.array([1], np.int32), np.array([1], np.int32), 2)
    with pytest.raises(ValueError):
        O.count(g, [0, 2], [1, 3], 1)  # second edge touches no mapped node
    with pytest.raises(ValueError):
        O.count(g, [0, 1], [1, 1], 1)  # self-loop
