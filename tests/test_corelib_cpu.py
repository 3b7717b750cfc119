"""The corelib module's host-side surface (the names system/tmine/core.py
imports from the reference's module), without a GPU."""
import os

import numpy as np
import pytest

from everest_b200 import capi, synth
from everest_b200.tmine import core
from oracle import oracle as O


def write_graph(path, u, v, t):
    synth.write_edge_text(str(path), u, v, t)


def test_module_names():
    for name in ("GPUWorker", "GPUWorkerLibManager", "SingleGPUExecution", "SingleGPUExecutionDiv",
                 "SingleGPURunBatch", "SingleGPUExecutionPause", "allCount", "MultiGPUExecutionNaive",
                 "MultiGPUExecutionDyn", "MultiGPUExecutionDynPause"):
        assert hasattr(core, name)
    for name in ("EdgeListLoader", "FeatureLoader", "GraphDataLoader", "HostGraphData", "HostMotifData",
                 "DeviceJobData", "MineJob", "MakeGraphDataManager", "divideList", "removeMinor",
                 "includeMinor", "SubPartitionList", "HostGraphDataList"):
        assert hasattr(core.data, name)


def test_edge_list_loader_and_cache(tmp_path):
    spec = synth.GraphSpec("cl-zipf", "zipf", 300, 5000, seed=2, t_max=9000)
    u, v, t = synth.generate(spec)
    perm = np.random.default_rng(0).permutation(u.size)
    p = tmp_path / "g.txt"
    write_graph(p, u[perm], v[perm], t[perm])
    e = core.data.EdgeListLoader(str(p))
    assert e.edgeListLength() == u.size
    cdir = tmp_path / "g"
    for f in ("U.cache", "V.cache", "T.cache", "IDS.cache"):
        assert (cdir / f).exists()
    ids = np.fromfile(cdir / "IDS.cache", dtype=np.int32)
    assert np.array_equal(ids, np.argsort(t[perm], kind="stable"))
    e2 = core.data.EdgeListLoader(str(p))  # from the cache
    assert e2.edgeListLength() == u.size
    f = core.data.FeatureLoader(e, "")
    assert f.edgeFeaturesLength() == 0
    gl = core.data.GraphDataLoader(e, f)
    hg = gl.createGraphData()
    assert hg.numEdges == u.size
    assert hg.totalBytes == 24 * hg.numEdges + 8 * (hg.numVertices + 1) + 4 * hg.numVertices
    assert (cdir / f"g-0-{u.size}" / "Eg").exists()
    hg2 = gl.createGraphData()  # from the per-range cache directory
    assert (hg2.numEdges, hg2.numVertices) == (hg.numEdges, hg.numVertices)
    part = gl.createGraphData(100, 900, False)
    assert part.numEdges == 800 and part.beg == 100 and part.end == 900


def test_feature_loader_follows_the_reference_mapping(tmp_path):
    """Edge i (time-sorted) takes rands[i]; the input vertex of rank r among
    the distinct ids takes rands[r] (src/core/gpu/data.cu:57-79,200-216); a
    relabeled vertex carries its input vertex's feature."""
    spec = synth.GraphSpec("cl-feat", "zipf", 400, 3000, seed=4, t_max=9000)
    u, v, t = synth.generate(spec)
    u = u * 7 + 11  # sparse, unordered input ids
    v = v * 7 + 11
    p = tmp_path / "g.txt"
    write_graph(p, u, v, t)
    rands = np.random.default_rng(1).integers(-10**9, 10**9, u.size + 50).astype(np.int32)
    rp = tmp_path / "rands.bin"
    rands.tofile(rp)
    e = core.data.EdgeListLoader(str(p))
    f = core.data.FeatureLoader(e, str(rp))
    ids = np.unique(np.concatenate([u, v]))
    assert f.edgeFeaturesLength() == u.size and f.verticesFeaturesLength() == ids.size
    hg = core.data.GraphDataLoader(e, f).createGraphData(0, 0, False)
    assert np.array_equal(np.asarray(hg.edgeFeatures), rands[: u.size])
    eg = np.asarray(hg.Eg).reshape(-1, 3)
    vf = np.asarray(hg.verticesFeatures)
    assert np.array_equal(vf[eg[:, 0]], rands[np.searchsorted(ids, u)])
    assert np.array_equal(vf[eg[:, 1]], rands[np.searchsorted(ids, v)])
    # the reference's feature caches, written beside the edge-list cache ...
    cdir = tmp_path / "g"
    assert np.array_equal(np.fromfile(cdir / "EdgesFeatures", np.int32), rands[: u.size])
    assert np.array_equal(np.fromfile(cdir / "VerticesFeaturesValue", np.int32), rands[: ids.size])
    assert np.array_equal(np.fromfile(cdir / "VerticesFeaturesMap", np.int32), ids)
    # ... and read back without the random-feature file
    f3 = core.data.FeatureLoader(e, "")
    hg3 = core.data.GraphDataLoader(e, f3).createGraphData(0, 0, False)
    assert np.array_equal(np.asarray(hg3.verticesFeatures), vf)
    assert np.array_equal(np.asarray(hg3.edgeFeatures), rands[: u.size])
    # a short file (and no cache) gives no features
    (tmp_path / "b").mkdir()
    write_graph(tmp_path / "b" / "g.txt", u, v, t)
    eb = core.data.EdgeListLoader(str(tmp_path / "b" / "g.txt"))
    rands[:10].tofile(rp)
    f2 = core.data.FeatureLoader(eb, str(rp))
    assert f2.edgeFeaturesLength() == 0 and f2.verticesFeaturesLength() == 0


def divide_list_restated(T, delta, num):
    """src/core/cpu/data.cc:345-369 restated in Python."""
    size = len(T)
    res = [[0, 0, 0] for _ in range(2 * num - 1)]
    chunk = size // num
    for i in range(num):
        res[i][0], res[i][1] = i * chunk, (i + 1) * chunk
    res[num - 1][1] = size
    res[num - 1][2] = res[num - 1][1] - res[num - 1][0]
    for i in range(num - 1):
        p = res[i][1]
        tt = int(T[p])
        lo = int(np.searchsorted(T, tt - delta, side="left")) - 1
        hi = int(np.searchsorted(T, tt + delta, side="left")) + 1
        res[i + num] = [lo, hi, p - lo]
        res[i][2] = lo - res[i][0]
    return res


def test_divide_list(tmp_path):
    spec = synth.GraphSpec("dl-zipf", "zipf", 300, 6000, seed=8, t_max=50_000)
    u, v, t = synth.generate(spec)
    p = tmp_path / "d.txt"
    write_graph(p, u, v, t)
    e = core.data.EdgeListLoader(str(p))
    for num in (1, 2, 3, 5):
        parts = core.data.divideList(e, 300, num)
        got = [[x.beg, x.end, x.n] for x in parts]
        assert got == divide_list_restated(t, 300, num)


def test_host_motif_data(tmp_path):
    p = tmp_path / "M4.txt"
    p.write_text("1 2 1\n2 3 2\n3 4 3\n4 1 4\n")
    m = core.data.HostMotifData(str(p))
    assert m.numEdges == 4 and m.numVertices == 4 and m.name == "M4"
    assert m.edges == [(0, 1, 1), (1, 2, 2), (2, 3, 3), (3, 0, 4)]
    # src/core/cpu/data.cc:416-446: (baseNode, constraintNode, mappedNodes, io, newNode)
    assert m.minfo == [(1, -2, 2, 1, True), (2, -3, 3, 1, True), (0, 3, 4, -1, False)]
    m2 = core.data.HostMotifData.fromText("2 3 1\n2 1 2\n3 4 3\n", "M2")
    assert m2.minfo == [(0, -2, 2, 1, True), (1, -3, 3, 1, True)]


def test_multi_gpu_refused_and_managers():
    with pytest.raises(ValueError):
        core.data.MakeGraphDataManager(0)
    dm = core.data.MakeGraphDataManager(1)
    with pytest.raises(ValueError):
        core.MultiGPUExecutionDyn(dm, 2)
    assert core.MultiGPUExecutionNaive(dm, 1).numDevice() == 1


def test_plugin_library_opens_without_gpu():
    from everest_b200.tmine import locations
    lm = core.GPUWorkerLibManager()
    lm.openLib(locations.dynLibPath())
    if capi.device_count() == 0:
        with pytest.raises(RuntimeError):
            lm.construct("EVX", 0)
    with pytest.raises(Exception):
        lm.construct("NOPE", 0)
    with pytest.raises(ValueError):
        lm.openLib("/tmp/not_a_plugin_name.so")
