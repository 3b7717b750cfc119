"""YAML query model of the drop-in driver (system/tmine/Query.py surface)."""
import pytest

from everest_b200.tmine import Query, utils


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_query_defaults_and_paths(tmp_path, monkeypatch):
    monkeypatch.setenv("EVX_MOTIF_ROOT", str(tmp_path))
    monkeypatch.setenv("EVX_GRAPH_ROOT", str(tmp_path))
    write(tmp_path, "M1.txt", "1 2 1\n2 3 2\n3 4 3\n")
    write(tmp_path, "g.txt", "0 1 1\n")
    q = Query.Query(write(tmp_path, "q.yaml", "pattern: M1.txt\ngraph: g.txt\nconstraints:\n  delta: 86400\n"
                                              "options:\n  gpu: 1\n"))
    assert q.pattern() == str(tmp_path / "M1.txt")
    assert q.graph() == str(tmp_path / "g.txt")
    assert q.constraints().delta() == 86400
    o = q.options()
    assert o.gpu() == 1 and not o.multigpu() and not o.enumerate() and o.flags() == 0
    assert o.opts["warpCentric"] and o.opts["warpBalancing"] and o.opts["tailExpansion"]


def test_query_enumerate_and_flags(tmp_path):
    q = Query.Query(write(tmp_path, "q.yaml", "pattern: a.txt\ngraph: b.txt\nconstraints: {delta: 5}\n"
                                              "options: {gpu: 1, enumerate: 1000, warpBalancing: False,"
                                              " tailExpansion: False}\n"))
    o = q.options()
    assert o.enumerate() and o.enumNum() == 1000
    assert o.flags() == 4 | 8


def test_query_constraints_compile_against_the_motif(tmp_path):
    q = Query.Query(write(tmp_path, "q.yaml", "pattern: a\ngraph: b\nconstraints: {delta: 5, temporal: [1, 2, 3], "
                                             "antiEdge: [False, False, True, False], node: 'f > 3', "
                                             "filter: 'e0 + e3 > 1'}\n"))
    c = q.constraints()
    assert c.isTemporal() and c.isAnti() and c.isFilter() and c.delta() == 5
    st = c.compile([0, 1, 2, 2], [1, 2, 0, 3]).to_struct()
    assert st.anti_mask == 4 and st.has_temporal and st.node_mode == 1 and st.has_filter
    for cons, mu, mv in (("{delta: 5, edge0: 'f > 1'}", [0, 1], [1, 2]),
                         ("{delta: 5, antiEdge: [False, True, False]}", [0, 1, 2], [1, 2, 0]),
                         ("{delta: 5, label: 3}", [0, 1], [1, 2])):
        q = Query.Query(write(tmp_path, "q1.yaml", f"pattern: a\ngraph: b\nconstraints: {cons}\n"))
        with pytest.raises(ValueError):
            q.constraints().compile(mu, mv)
    with pytest.raises(ValueError):
        Query.Query(write(tmp_path, "q2.yaml", "pattern: a\ngraph: b\nconstraints: {}\n"))


def test_inspect_motif_and_lib_names(tmp_path):
    p = write(tmp_path, "M3.txt", "1 2 1 \n2 3 2\n3 4 3\n4 2 4\n")
    assert utils.InspectMotif(p) == ([2, 3, 4], 2, 4)
    assert utils.libFileToLibName("/x/y/libEVX.so") == "EVX"
    assert utils.libNameToLibFile("DYN") == "libDYN.so"
