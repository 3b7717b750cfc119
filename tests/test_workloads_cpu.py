"""Query mixes of the batch / serve measurements and the equality rule the
two arms are compared by (CPU only)."""
import numpy as np

import bench_modes
from everest_b200 import synth, workloads


def test_batch_and_serve_mixes_are_seeded_and_in_range():
    a, b = workloads.batch_queries(), workloads.batch_queries()
    assert a == b and len(a) == 64
    E = synth.SPECS["bursty-2.6m-36m"].num_edges
    for q in a:
        assert len(q["mu"]) in (3, 4) and q["delta"] in (3600, 86400, 604800)
        assert 0 <= q["beg"] < q["end"] <= E and q["end"] - q["beg"] <= 1_000_000
        assert max(q["mu"] + q["mv"]) + 1 <= 4 and q["cap"] == 0
    s = workloads.serve_queries(n=500)
    assert s == workloads.serve_queries(n=500)
    caps = [q["cap"] for q in s if q["cap"]]
    assert 0.1 < len(caps) / len(s) < 0.3 and all(1e4 <= c <= 1e6 for c in caps)
    assert all(600 <= q["delta"] <= 604800 and 3 <= len(q["mu"]) <= 5 for q in s)
    assert {q["graph"] for q in s} == {"bursty-1.1m-7.8m", "bursty-6m-63m"}


def test_result_equality_rule():
    q_count, q_enum = {"cap": 0}, {"cap": 3}
    rows = np.array([[1, 2], [3, 4]], np.int32)
    same = bench_modes._same
    assert same((5, False, None), (5, False, None), q_count)
    assert not same((5, False, None), (6, False, None), q_count)
    assert same((9, True, None), (None, True, None), q_count)        # limited in both arms
    assert not same((9, True, None), (9, False, None), q_count)      # limited in one arm only
    assert same((2, False, rows), (2, False, rows[::-1]), q_enum)   # row order is free
    assert not same((2, False, rows), (2, False, rows[:1].repeat(2, 0)), q_enum)
    capped = np.arange(6, dtype=np.int32).reshape(3, 2)
    assert same((10, False, capped), (12, False, capped[::-1]), q_enum)  # both past the cap
