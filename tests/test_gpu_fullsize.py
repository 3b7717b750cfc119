"""Full-size enumeration (C4: the 4-cycle 0->1->2->3->0 on the 2.6M-node /
36M-edge graph, delta 86400, cap 1e6) checked against the oracle where the
oracle enumerates fully, and the exact total against the reference's own
generated kernel (tests/golden/full_size_counts.json)."""
import json
import os

import numpy as np
import pytest

from everest_b200 import capi, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
MU, MV, DELTA, CAP = [0, 1, 2, 3], [1, 2, 3, 0], 86400, 1_000_000


def _keys(rows):
    """Exact 16-byte keys of int64 rows of four edge ids (ids < 2^31)."""
    r = rows.astype(np.int64)
    k = np.ascontiguousarray(np.stack([(r[:, 0] << 32) | r[:, 1], (r[:, 2] << 32) | r[:, 3]], axis=1))
    return k.view("V16").ravel()


@pytest.fixture(scope="module")
def c4():
    spec = synth.SPECS["bursty-2.6m-36m"]
    u, v, t = synth.load_or_generate(spec.name)
    g = O.Graph(u, v, t, spec.num_nodes)
    dg = capi.DeviceGraph(capi.graph_build_host(u, v, t), 0)
    w = capi.Worker(0)
    yield g, dg, w
    w.close()
    dg.free()


def test_capped_rows_are_oracle_rows(c4):
    g, dg, w = c4
    with open(os.path.join(HERE, "golden", "full_size_counts.json")) as f:
        total_ref = json.load(f)["bursty-2.6m-36m"]["4-cycle delta 86400"]
    w.take(dg, MU, MV, DELTA, 0, -1, CAP, capi.FLAG_EXACT_TOTAL)
    assert w.run() == total_ref  # the exact total past the cap
    w.take(dg, MU, MV, DELTA, 0, -1, CAP)
    assert w.run() >= CAP
    rows = w.enum_rows(CAP).astype(np.int64)
    assert rows.shape == (CAP, 4)
    assert len(np.unique(rows, axis=0)) == CAP  # no duplicates
    # every row is a match the oracle finds among the roots the rows start from
    hi = int(rows[:, 0].max()) + 1
    tot, _ = O.count(g, MU, MV, DELTA, roots=(0, hi))
    want, tot2 = O.enumerate_rows(g, MU, MV, DELTA, tot, roots=(0, hi))
    assert tot2 == tot and want.shape[0] == tot
    ws = np.sort(_keys(want))
    k = _keys(rows)
    pos = np.searchsorted(ws, k)
    pos[pos >= ws.size] = 0
    hit = ws[pos] == k
    assert hit.all(), f"{int((~hit).sum())} rows are not oracle matches"
    print(f"\n4-cycle, 36M edges: {CAP} capped rows drawn from roots [0, {hi}), all among the oracle's {tot}")


def test_rows_equal_oracle_on_a_root_range(c4):
    g, dg, w = c4
    r0, r1 = 18_000_000, 18_400_000
    tot, _ = O.count(g, MU, MV, DELTA, roots=(r0, r1))
    assert 0 < tot <= 20_000_000
    want, _ = O.enumerate_rows(g, MU, MV, DELTA, tot, roots=(r0, r1))
    w.take(dg, MU, MV, DELTA, r0, r1, tot + 16)
    assert w.run() == tot
    got = w.enum_rows(tot + 16)
    assert sorted(map(tuple, got.tolist())) == sorted(map(tuple, want.tolist()))
    print(f"\n4-cycle, 36M edges, roots [{r0}, {r1}): {tot} rows equal to the oracle's")
