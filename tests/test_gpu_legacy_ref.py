"""The reference's own legacy Baseline search kernel, built for sm_100a from
its sources (oracle/ref_gpu_driver.cu), against this library on the same
graphs: every count equal.  The reference's kernel runs one thread per root
and no load balancing; the times of both are printed (pytest -s) as the
kernel-level comparison on the same GPU."""
import pytest

from everest_b200 import capi, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    if O.ref_gpu_lib() is None:
        pytest.skip("the reference's Baseline kernel was not built (needs the reference tree at build time)")
    return O


def _ours(w, dg, mu, mv, d):
    best = None
    for _ in range(2):
        w.take(dg, mu, mv, d)
        c = w.run()
        ms = w.last_stats()["device_ms"]
        best = ms if best is None else min(best, ms)
    return c, best


def test_reference_kernel_counts_equal_ours(ref):
    spec = synth.GraphSpec("legacy-bursty", "bursty", 50_000, 400_000, seed=71, t_span=12_000_000)
    u, v, t = synth.generate(spec)
    g = O.Graph(u, v, t, spec.num_nodes)
    dg = capi.DeviceGraph(capi.graph_build_host(u, v, t), 0)
    w = capi.Worker(0)
    qs = [([a for a, b in p], [b for a, b in p], 86400) for p in synth.three_edge_patterns()]
    qs += [([0, 1, 2, 3], [1, 2, 3, 0], 86400), ([0, 0, 0, 0], [1, 2, 3, 4], 3600)]
    t_ref = t_ours = 0.0
    for mu, mv, d in qs:
        c_ref, ms_ref = O.ref_gpu_count(g, mu, mv, d)
        c, ms = _ours(w, dg, mu, mv, d)
        assert c == c_ref, (mu, mv, d, c, c_ref)
        t_ref += ms_ref
        t_ours += ms
    print(f"\n{len(qs)} queries on a 400k-edge bursty graph: reference Baseline kernel {t_ref:.2f} ms, "
          f"this library {t_ours:.2f} ms ({t_ref / max(t_ours, 1e-9):.1f}x)")
    w.close()
    dg.free()


def test_reference_kernel_on_the_bench_graph(ref):
    # the 7.8M-edge bench graph, the 36 three-edge motifs at delta 86400:
    # counts equal, times printed
    from everest_b200 import workloads
    u, v, t = synth.load_or_generate("bursty-1.1m-7.8m")
    g = O.Graph(u, v, t, synth.SPECS["bursty-1.1m-7.8m"].num_nodes)
    dg = capi.DeviceGraph(capi.graph_build_host(u, v, t), 0)
    w = capi.Worker(0)
    t_ref = t_ours = 0.0
    for q in workloads.queries("bursty-7.8m-3edge"):
        c_ref, ms_ref = O.ref_gpu_count(g, q["mu"], q["mv"], q["delta"], reps=1)
        c, ms = _ours(w, dg, q["mu"], q["mv"], q["delta"])
        assert c == c_ref, (q["name"], c, c_ref)
        t_ref += ms_ref
        t_ours += ms
    print(f"\n36 three-edge motifs on the 7.8M-edge graph: reference Baseline kernel {t_ref:.1f} ms, "
          f"this library (default launch parameters) {t_ours:.1f} ms ({t_ref / max(t_ours, 1e-9):.1f}x)")
    w.close()
    dg.free()
