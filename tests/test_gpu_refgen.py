"""The search kernel the reference generates per query (KernelGen with
warpCentric, warpBalancing and tailExpansion on, the configuration Everest
ships), built for sm_100a by baseline/refgen.py, run through its own
GPUWorker on the same B200 as this library.

It is pinned first to the golden fixtures (the reference's Baseline body and
the oracle), then used as the full-size check of this library: the 36
three-edge motifs on the 7.8M-edge graph, the 4-cycle total on the 36M-edge
graph, and 16 queries of the 64-query batch mix.  Times of both are printed
(pytest -s)."""
import json
import os

import numpy as np
import pytest

from baseline import refgen as R
from everest_b200 import capi, synth, workloads
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _need(pats):
    missing = [R.query_key(mu, mv) for mu, mv in pats if not R.available(mu, mv)]
    if missing:
        pytest.skip(f"generated kernels not built ({len(missing)} missing; python -m baseline.refgen build)")


def _ours(w, dg, mu, mv, d, beg=0, end=-1, reps=2):
    best = None
    for _ in range(reps):
        w.take(dg, mu, mv, d, beg, end)
        c = w.run()
        ms = w.last_stats()["device_ms"]
        best = ms if best is None else min(best, ms)
    return c, best


def test_generated_kernel_matches_golden_counts():
    with open(os.path.join(HERE, "golden", "golden.json")) as f:
        golden = json.load(f)
    _need({(tuple(c["mu"]), tuple(c["mv"])) for c in golden["cases"]})
    z = np.load(os.path.join(HERE, "golden", "small_graphs.npz"))
    by_graph = {}
    for c in golden["cases"]:
        by_graph.setdefault(c["graph"], []).append(c)
    n = 0
    for gname, cases in by_graph.items():
        g = O.Graph(z[f"{gname}_u"], z[f"{gname}_v"], z[f"{gname}_t"], int(z[f"{gname}_V"][0]))
        rg = R.RefGraph.from_oracle_graph(g)
        for c in cases:
            rb, re_ = c.get("roots", [0, -1])
            got, _ = R.count(rg, c["mu"], c["mv"], c["delta"], rb, re_)
            assert got == c["count"], (gname, c["motif"], c["delta"], rb, re_, got, c["count"])
            n += 1
        rg.free()
    assert n == len(golden["cases"])


def test_generated_kernel_on_the_200k_triangle():
    with open(os.path.join(HERE, "golden", "golden.json")) as f:
        tri = json.load(f)["full_zipf"]["triangle"]
    _need([(tri["mu"], tri["mv"])])
    spec = synth.SPECS["zipf-10k-200k"]
    u, v, t = synth.load_or_generate(spec.name)
    rg = R.RefGraph.from_oracle_graph(O.Graph(u, v, t, spec.num_nodes))
    got, ms = R.count(rg, tri["mu"], tri["mv"], tri["delta"], reps=3)
    rg.free()
    assert got == tri["count"]
    print(f"\n200k-edge triangle, delta 3600: generated kernel {min(ms):.3f} ms, count {got}")


def _full_size(graph_name, queries, label):
    _need([(q["mu"], q["mv"]) for q in queries])
    spec = synth.SPECS[graph_name]
    u, v, t = synth.load_or_generate(spec.name)
    rg = R.RefGraph.from_oracle_graph(O.Graph(u, v, t, spec.num_nodes))
    dg = capi.DeviceGraph(capi.graph_build_host(u, v, t), 0)
    w = capi.Worker(0)
    t_ref = t_ours = 0.0
    rows = []
    try:
        for q in queries:
            beg, end = q.get("beg", 0), q.get("end", -1)
            c_ref, ms_ref = R.count(rg, q["mu"], q["mv"], q["delta"], beg, end, reps=1)
            c, ms = _ours(w, dg, q["mu"], q["mv"], q["delta"], beg, end)
            assert c == c_ref, (q["name"], c, c_ref)
            t_ref += ms_ref[0]
            t_ours += ms
            rows.append((q["name"], c, ms_ref[0], ms))
    finally:
        w.close()
        dg.free()
        rg.free()
    print(f"\n{label}: generated kernel {t_ref:.1f} ms (host time around run()), this library "
          f"{t_ours:.1f} ms (device time, default launch parameters): {t_ref / max(t_ours, 1e-9):.1f}x")
    for name, c, a, b in rows:
        print(f"  {name}: count {c}  generated {a:.2f} ms  ours {b:.2f} ms")
    return rows


def test_generated_kernel_36_three_edge_motifs():
    qs = workloads.queries("bursty-7.8m-3edge")
    want = {r["name"]: r["count"] for r in
            json.load(open(os.path.join(HERE, "golden", "workload_stats.json")))["bursty-7.8m-3edge"]["queries"]}
    rows = _full_size("bursty-1.1m-7.8m", qs, "36 three-edge motifs, 7.8M edges, delta 86400")
    for name, c, _, _ in rows:
        assert c == want[name]


def _fixture():
    with open(os.path.join(HERE, "golden", "full_size_counts.json")) as f:
        return json.load(f)["bursty-2.6m-36m"]


def test_generated_kernel_4cycle_36m():
    q = {"name": "4-cycle", "mu": [0, 1, 2, 3], "mv": [1, 2, 3, 0], "delta": 86400}
    rows = _full_size("bursty-2.6m-36m", [q], "4-cycle, 36M edges, delta 86400")
    assert rows[0][1] == _fixture()["4-cycle delta 86400"]


def test_generated_kernel_serve_slice():
    """16 count queries of the serving stream on both resident graphs."""
    qs = workloads.refgen_serve_slice()
    assert len(qs) == 16 and all(q["cap"] == 0 for q in qs)
    for gname in sorted({q["graph"] for q in qs}):
        _full_size(gname, [q for q in qs if q["graph"] == gname], f"serving-stream slice on {gname}")


def test_generated_kernel_batch_mix_slice():
    qs = workloads.refgen_batch_slice()
    assert len(qs) == 16
    rows = _full_size("bursty-2.6m-36m", qs, "16 queries of the 64-query batch mix, 36M edges")
    fix = _fixture().get("batch slice")
    if fix is not None:
        for name, c, _, _ in rows:
            assert c == fix[name]["count"], name
