"""The reference's legacy ablation plugins (plugins/GPUWorker{U0,U1,U1B,U2,
U3,U3B}.cu, the optimisation ladder of its README's "Figure 10"), built for
sm_100a by baseline/legacy.py and run through their own GPUWorker on the
same B200 as this library and the reference's generated kernel: every count
equal; the times of each (host time around run(), the reference's
convention) are printed as the ablation table (pytest -s)."""
import pytest

from baseline import legacy as L
from baseline import refgen as R
from everest_b200 import capi, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _need():
    missing = [p for p in L.PLUGINS if not L.available(p)]
    if missing:
        pytest.skip(f"legacy plugins not built ({missing}; python -m baseline.legacy build)")


def _table(graph_name_or_spec, queries, label):
    _need()
    if isinstance(graph_name_or_spec, synth.GraphSpec):
        spec = graph_name_or_spec
        u, v, t = synth.generate(spec)
    else:
        spec = synth.SPECS[graph_name_or_spec]
        u, v, t = synth.load_or_generate(spec.name)
    g = O.Graph(u, v, t, spec.num_nodes)
    rg = R.RefGraph.from_oracle_graph(g)
    dg = capi.DeviceGraph(capi.graph_build_host(u, v, t), 0)
    w = capi.Worker(0)
    gen_ok = all(R.available(mu, mv) for mu, mv, _ in queries)
    times = {p: 0.0 for p in L.PLUGINS}
    times["generated"] = 0.0
    times["this library"] = 0.0
    try:
        for mu, mv, d in queries:
            w.take(dg, mu, mv, d)
            want = w.run()
            import time
            t0 = time.perf_counter()
            w.take(dg, mu, mv, d)
            assert w.run() == want
            times["this library"] += (time.perf_counter() - t0) * 1e3
            for p in L.PLUGINS:
                c, ms = L.count(p, rg, mu, mv, d)
                assert c == want, (p, mu, mv, d, c, want)
                times[p] += ms[0]
            if gen_ok:
                c, ms = R.count(rg, mu, mv, d)
                assert c == want, ("generated", mu, mv, d, c, want)
                times["generated"] += ms[0]
    finally:
        w.close()
        dg.free()
        rg.free()
    print(f"\n{label}: host ms around run(), summed over {len(queries)} queries")
    for k, ms in times.items():
        if k == "generated" and not gen_ok:
            continue
        print(f"  {k:>13}: {ms:9.1f} ms")
    return times


def test_legacy_plugins_equal_counts_400k():
    spec = synth.GraphSpec("legacy-bursty", "bursty", 50_000, 400_000, seed=71, t_span=12_000_000)
    qs = [([a for a, b in p], [b for a, b in p], 86400) for p in synth.three_edge_patterns()]
    qs += [([0, 1, 2, 3], [1, 2, 3, 0], 86400), ([0, 0, 0, 0], [1, 2, 3, 4], 3600),
           ([0, 1, 1, 2], [1, 2, 0, 0], 86400), ([0, 1, 2, 3, 1], [1, 2, 3, 1, 4], 3600)]
    _table(spec, qs, "legacy plugins, 400k-edge bursty graph")


def test_legacy_plugins_on_the_bench_graph():
    qs = [([a for a, b in p], [b for a, b in p], 86400) for p in synth.three_edge_patterns()]
    _table("bursty-1.1m-7.8m", qs, "legacy plugins, 36 three-edge motifs on the 7.8M-edge graph")
