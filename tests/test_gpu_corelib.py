"""The drop-in surface end to end on the GPU: YAML query -> tmine driver ->
corelib -> getWorker plugin -> sm_100a kernels, checked against the oracle."""
import numpy as np
import pytest

from everest_b200 import synth
from everest_b200.tmine import core, frontend, locations
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def inputs(tmp_path_factory):
    d = tmp_path_factory.mktemp("inputs")
    spec = synth.GraphSpec("e2e-zipf", "zipf", 600, 25_000, seed=21, t_max=400_000)
    u, v, t = synth.generate(spec)
    perm = np.random.default_rng(2).permutation(u.size)  # file lines out of time order
    synth.write_edge_text(str(d / "g.txt"), u[perm], v[perm], t[perm])
    (d / "M4.txt").write_text("1 2 1\n2 3 2\n3 4 3\n4 1 4\n")
    (d / "T.txt").write_text("1 2 1\n2 3 2\n3 1 3\n")
    order = np.argsort(t[perm], kind="stable")   # sorted edge i = line order[i]
    g = O.Graph(u[perm][order], v[perm][order], t[perm][order], spec.num_nodes)
    return d, g, order


def yaml(d, name, pattern, delta, extra=""):
    p = d / name
    p.write_text(f"pattern: {pattern}\ngraph: g.txt\nconstraints:\n  delta: {delta}\n"
                 f"options:\n  gpu: 1\n{extra}")
    return str(p)


def test_single_query_count(inputs, monkeypatch):
    d, g, order = inputs
    monkeypatch.setenv("EVX_MOTIF_ROOT", str(d))
    monkeypatch.setenv("EVX_GRAPH_ROOT", str(d))
    lines = []
    cnt, us, sec = frontend.MiningSingle(yaml(d, "q1.yaml", "M4.txt", 5000)).run(
        out=lambda *a, **k: lines.append(" ".join(map(str, a))))
    want, _ = O.count(g, [0, 1, 2, 3], [1, 2, 3, 0], 5000)
    assert cnt == want and want > 0
    assert lines[0] == "@@@ [output starts]" and lines[-1] == "@@@ [output ends]"
    assert lines[1].split(",")[0] == str(want)


def test_batch_of_queries_one_resident_graph(inputs, monkeypatch):
    d, g, order = inputs
    monkeypatch.setenv("EVX_MOTIF_ROOT", str(d))
    monkeypatch.setenv("EVX_GRAPH_ROOT", str(d))
    m = frontend.Mining(str(d / "g.txt"), 1)
    for pat, mu, mv, delta in (("T.txt", [0, 1, 2], [1, 2, 0], 3000), ("M4.txt", [0, 1, 2, 3], [1, 2, 3, 0], 8000),
                               ("T.txt", [0, 1, 2], [1, 2, 0], 20000)):
        cnt = m.run(yaml(d, "qb.yaml", pat, delta), out=lambda *a, **k: None)[0]
        assert cnt == O.count(g, mu, mv, delta)[0]


def test_enumerate_query_rows_are_original_line_ids(inputs, monkeypatch):
    d, g, order = inputs
    monkeypatch.setenv("EVX_MOTIF_ROOT", str(d))
    monkeypatch.setenv("EVX_GRAPH_ROOT", str(d))
    want_rows, total = O.enumerate_rows(g, [0, 1, 2], [1, 2, 0], 4000, 10 ** 6)
    assert 0 < total < 10 ** 6
    res = frontend.MiningSingle(yaml(d, "q2.yaml", "T.txt", 4000, f"  enumerate: {total + 10}\n")).run(
        out=lambda *a, **k: None)
    cnt, rows = res[0], res[3]
    assert cnt == total
    want = sorted(order[want_rows].tolist())
    assert sorted(rows.tolist()) == want


def test_legacy_corelib_flow(inputs):
    """The sequence system/legacy.py drives through corelib."""
    d, g, order = inputs
    e = core.data.EdgeListLoader(str(d / "g.txt"))
    f = core.data.FeatureLoader(e, "")
    gl = core.data.GraphDataLoader(e, f)
    hg = gl.createGraphData()
    hm = core.data.HostMotifData(str(d / "M4.txt"))
    dm = core.data.MakeGraphDataManager(1)
    lm = core.GPUWorkerLibManager()
    lm.openLib(locations.dynLibPath())
    w = lm.construct("EVX", 0)
    ex = core.SingleGPUExecution(dm)
    ex.setHostGraph(hg)
    ex.setHostMotif(hm)
    ex.setWorker(w)
    r = ex.run(5000)
    want, _ = O.count(g, [0, 1, 2, 3], [1, 2, 3, 0], 5000)
    assert r == w.count() == want
    assert w.time() > 0
    w.clear_time()
    assert w.time() == 0
    ex2 = core.SingleGPUExecutionDiv(dm, 0, 7)
    ex2.setHostGraph(hg)
    ex2.setHostMotif(hm)
    ex2.setWorker(w)
    assert ex2.run(5000) == want
    assert core.allCount([w]) == want
    del w


def test_constrained_query_end_to_end(tmp_path, monkeypatch):
    """A YAML query with node predicates, temporal gaps, an anti-edge and a
    filter, features from a random-feature file, through the tmine driver."""
    from everest_b200.constraints import Constraints
    spec = synth.GraphSpec("e2e-cons", "zipf", 500, 20_000, seed=23, t_max=200_000)
    u, v, t = synth.generate(spec)
    perm = np.random.default_rng(5).permutation(u.size)
    synth.write_edge_text(str(tmp_path / "g.txt"), u[perm], v[perm], t[perm])
    rands = np.random.default_rng(6).integers(0, 10, u.size + 10).astype(np.int32)
    rands.tofile(tmp_path / "rands.bin")
    (tmp_path / "M4-A.txt").write_text("1 2 1\n2 3 2\n3 1 3\n3 4 4\n4 1 5\n")
    cons = {"delta": 20_000, "node0": "f > 2", "node1": "f < 8", "node2": "f > 1", "node3": "f != 5",
            "antiEdge": [False, False, True, False, False], "temporal": [10_000, 15_000, 15_000, 10_000],
            "filter": "(e0 + e1 + e3) > 6"}
    q = tmp_path / "q.yaml"
    q.write_text("pattern: M4-A.txt\ngraph: g.txt\nconstraints:\n"
                 + "".join(f"  {k}: {v!r}\n" if isinstance(v, str) else f"  {k}: {v}\n" for k, v in cons.items())
                 + "options:\n  gpu: 1\n")
    monkeypatch.setenv("EVX_MOTIF_ROOT", str(tmp_path))
    monkeypatch.setenv("EVX_GRAPH_ROOT", str(tmp_path))
    monkeypatch.setenv("EVX_RAND_FILE", str(tmp_path / "rands.bin"))
    cnt = frontend.MiningSingle(str(q)).run(out=lambda *a, **k: None)[0]
    order = np.argsort(t[perm], kind="stable")
    us, vs, ts = u[perm][order], v[perm][order], t[perm][order]
    ids = np.unique(np.concatenate([u, v]))
    V = int(ids.max()) + 1
    nf = np.zeros(V, np.int32)
    nf[ids] = rands[: ids.size]
    mu, mv = [0, 1, 2, 2, 3], [1, 2, 0, 3, 0]
    c = Constraints.from_yaml(cons, mu, mv).to_struct()
    want = O.count_constrained(O.Graph(us, vs, ts, V), mu, mv, 20_000, c, nf, rands[: u.size])
    assert cnt == want and want > 0
