"""Host-side C-ABI functions (no GPU): symbol exports, edge-list parsing,
graph building, motif decoding, error codes."""
import ctypes
import os
import re

import numpy as np
import pytest

from everest_b200 import capi, synth
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            with open(os.path.join(inc, f)) as fh:
                names += re.findall(r"EVX_API\s+[\w\s\*]+?\b(evx_\w+)\s*\(", fh.read())
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 24
    L = capi.lib()
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(capi.EXPORTS) | {"evx_count_static"}


def test_edgelist_parse_stable_sort(tmp_path):
    rng = np.random.default_rng(3)
    n = 5000
    u = rng.integers(0, 300, n)
    v = rng.integers(0, 300, n)
    t = rng.integers(0, 400, n)  # many ties
    p = tmp_path / "g.txt"
    with open(p, "w") as f:
        for a, b, c in zip(u, v, t):
            f.write(f"{a} {b} {c}\n")
        f.write("\n")  # trailing blank line is skipped
    pu, pv, pt, ids = capi.edgelist_parse(str(p))
    order = np.argsort(t, kind="stable")
    assert np.array_equal(ids, order)
    assert np.array_equal(pt, t[order]) and np.array_equal(pu, u[order]) and np.array_equal(pv, v[order])


def test_edgelist_parse_large_parallel(tmp_path):
    spec = synth.GraphSpec("parse-zipf", "zipf", 2000, 300_000, seed=9, t_max=100_000)
    u, v, t = synth.generate(spec)
    rng = np.random.default_rng(1)
    perm = rng.permutation(u.size)  # shuffle lines: the parser must restore time order
    p = tmp_path / "big.txt"
    synth.write_edge_text(str(p), u[perm], v[perm], t[perm])
    pu, pv, pt, ids = capi.edgelist_parse(str(p))
    order = np.argsort(t[perm], kind="stable")
    assert np.array_equal(ids, order)
    assert np.array_equal(pt, t[perm][order])


def test_graph_build_host_matches_oracle_csr():
    spec = synth.GraphSpec("csr-zipf", "zipf", 500, 20_000, seed=4)
    u, v, t = synth.generate(spec)
    h = capi.graph_build_host(u, v, t)
    g = O.Graph(u, v, t, spec.num_nodes)
    eg = h.eg.reshape(-1, 3)
    assert h.num_edges == u.size
    assert np.array_equal(eg[:, 2], t)
    # relabeled ids map back to original ids consistently
    back = {}
    for nu, ou in zip(eg[:, 0], u):
        assert back.setdefault(int(nu), int(ou)) == int(ou)
    for nv, ov in zip(eg[:, 1], v):
        assert back.setdefault(int(nv), int(ov)) == int(ov)
    for x in range(h.num_vertices):
        ox = back[x]
        assert np.array_equal(h.out_v[h.out_r[x]:h.out_r[x + 1]], g.out_eid[g.out_off[ox]:g.out_off[ox + 1]])
        assert np.array_equal(h.in_v[h.in_r[x]:h.in_r[x + 1]], g.in_eid[g.in_off[ox]:g.in_off[ox + 1]])
    assert np.array_equal(h.euid, np.arange(u.size))


def test_graph_build_host_range_and_ids():
    u = np.array([5, 7, 5, 9], np.int32)
    v = np.array([7, 9, 9, 5], np.int32)
    t = np.array([1, 1, 2, 3], np.int32)
    ids = np.array([10, 11, 12, 13], np.int32)
    h = capi.graph_build_host(u, v, t, ids, beg=1, end=4)
    assert h.num_edges == 3 and h.num_vertices == 3
    assert list(h.euid) == [11, 12, 13]
    with pytest.raises(capi.EvxError):
        capi.graph_build_host(u, v, np.array([3, 1, 2, 3], np.int32))  # not time-sorted


def test_motif_parse_matches_oracle():
    texts = ["1 2 1 \n2 3 2\n3 4 3\n4 2 4\n", "2 3 1\n2 1 2\n3 4 3\n", "5 9 3\n9 5 1\n5 7 2\n",
             "1 2 1\n\n2 3 2\n"]
    for tx in texts:
        mu, mv, nn = capi.motif_parse_text(tx)
        omu, omv = O.parse_motif(tx)
        assert (mu, mv) == (omu, omv)
        assert nn == max(max(mu), max(mv)) + 1


def test_motif_parse_errors(tmp_path):
    with pytest.raises(capi.EvxError) as ei:
        capi.motif_parse(str(tmp_path / "missing.txt"))
    assert ei.value.code == -5
    with pytest.raises(capi.EvxError) as ei:
        capi.motif_parse_text("1 2 x\n")
    assert ei.value.code == -1
    with pytest.raises(capi.EvxError):
        capi.motif_parse_text("".join(f"{i} {i+1} {i}\n" for i in range(9)))
    with pytest.raises(capi.EvxError):
        capi.motif_parse_text("")


def test_edgelist_missing_file():
    with pytest.raises(capi.EvxError) as ei:
        capi.edgelist_parse("/nonexistent/graph.txt")
    assert ei.value.code == -5


def test_no_device_errors_on_cpu_host():
    if capi.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(capi.EvxError) as ei:
        capi.Worker(0)
    assert ei.value.code == -8
    h = capi.graph_build_host(np.array([0], np.int32), np.array([1], np.int32), np.array([1], np.int32))
    with pytest.raises(capi.EvxError) as ei:
        capi.DeviceGraph(h, 0)
    assert ei.value.code in (-8, -1)


def test_upload_validation_rejects_bad_arrays():
    """Arrays that would send the packing kernels out of bounds are rejected
    on the host before anything reaches the device."""
    h = capi.graph_build_host(np.array([0, 1], np.int32), np.array([1, 0], np.int32),
                              np.array([1, 2], np.int32))
    h.out_v = h.out_v.copy()
    h.out_v[0] = 7  # edge id out of range
    with pytest.raises(capi.EvxError) as ei:
        capi.DeviceGraph(h, 0)
    assert ei.value.code in (-1, -8)
