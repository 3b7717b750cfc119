"""Named benchmark workloads (synthetic stand-ins for the reference's
SNAP / ethereum graphs, which are not available offline).

Each workload is a graph from ``synth.SPECS`` plus a list of queries
(relabeled motif edges, delta, count or enumerate cap)."""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import synth

WORKLOADS: Dict[str, dict] = {
    # 10k nodes / 200k edges, triangle 0->1->2->0, delta 3600, count
    "zipf-200k-triangle": {"graph": "zipf-10k-200k", "kind": "triangle", "delta": 3600},
    # 1.1M nodes / 7.8M edges, every connected 3-edge pattern on 2-3 nodes
    # (36 by rule), each run separately, delta 86400, count
    "bursty-7.8m-3edge": {"graph": "bursty-1.1m-7.8m", "kind": "three_edge", "delta": 86400},
    # the same graph, the 4-cycle 0->1->2->3->0, delta 86400, count
    "bursty-7.8m-4cycle": {"graph": "bursty-1.1m-7.8m", "kind": "four_cycle", "delta": 86400},
}


def queries(name: str) -> List[dict]:
    wl = WORKLOADS[name]
    if wl["kind"] == "triangle":
        return [{"name": "triangle", "mu": [0, 1, 2], "mv": [1, 2, 0], "delta": wl["delta"]}]
    if wl["kind"] == "four_cycle":
        return [{"name": "4-cycle", "mu": [0, 1, 2, 3], "mv": [1, 2, 3, 0], "delta": wl["delta"]}]
    if wl["kind"] == "three_edge":
        out = []
        for i, p in enumerate(synth.three_edge_patterns()):
            out.append({"name": f"3e-{i:02d}", "mu": [a for a, b in p], "mv": [b for a, b in p],
                        "delta": wl["delta"]})
        return out
    raise KeyError(name)


# ------------------------------------------------- batch and serving mixes --

def mixed_queries(n: int, seed: int, edge_range: Tuple[int, int], node_range: Tuple[int, int],
                  graphs: Sequence[Tuple[str, int]], window: int, deltas: Sequence[int] = (),
                  delta_range: Tuple[int, int] = (0, 0), enum_frac: float = 0.0,
                  cap_range: Tuple[float, float] = (1e4, 1e6)) -> List[dict]:
    """``n`` seeded queries over resident graphs.

    Each query: a random connected pattern (``synth.random_patterns``, edges
    and nodes drawn from the inclusive ranges), a graph (round robin over
    ``graphs`` = [(name, num_edges)]), a root window of ``window`` consecutive
    edge ids at a uniform random start (the reference's MineJob(data, delta,
    beg, end) root range; a window of edges is a window of time, the edge
    list being sorted by timestamp), delta from ``deltas`` round robin or
    log-uniform in ``delta_range``, and with probability ``enum_frac`` an
    enumeration with a cap log-uniform in ``cap_range`` (0 = count)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    pats = synth.random_patterns(n, edge_range, node_range, seed=seed) if n <= 200 else \
        synth.random_patterns(200, edge_range, node_range, seed=seed)
    out = []
    for i in range(n):
        p = pats[int(rng.integers(0, len(pats)))] if n > len(pats) else pats[i]
        gname, E = graphs[i % len(graphs)]
        beg = int(rng.integers(0, max(1, E - window)))
        if deltas:
            d = int(deltas[i % len(deltas)])
        else:
            d = int(np.exp(rng.uniform(np.log(delta_range[0]), np.log(delta_range[1]))))
        cap = 0
        if enum_frac and rng.random() < enum_frac:
            cap = int(np.exp(rng.uniform(np.log(cap_range[0]), np.log(cap_range[1]))))
        out.append({"graph": gname, "mu": [a for a, b in p], "mv": [b for a, b in p], "delta": d,
                    "beg": beg, "end": min(E, beg + window), "cap": cap})
    return out


def batch_queries(window: int = 1_000_000, n: int = 64) -> List[dict]:
    """64 queries mixing 3- and 4-edge patterns on 2-4 nodes, delta cycling
    through {3600, 86400, 604800}, on the 2.6M-node / 36M-edge graph."""
    spec = synth.SPECS["bursty-2.6m-36m"]
    return mixed_queries(n, 3, (3, 4), (2, 4), [(spec.name, spec.num_edges)], window,
                         deltas=(3600, 86400, 604800))


# The 16 queries of the 64-query mix whose search over the whole 36M-edge
# graph is cheapest (1.6-6 ms each for this library on a B200; of the other
# 48, 29 examine more than 3e9 adjacency records each).
BATCH_SLICE = (36, 63, 30, 3, 10, 48, 19, 0, 6, 1, 24, 39, 51, 49, 57, 15)


def refgen_batch_slice() -> List[dict]:
    """BATCH_SLICE of the 64-query batch mix over every root of the graph:
    the full-size slice the reference's generated kernel checks."""
    qs = batch_queries()
    return [dict(qs[i], name=f"batch-{i:02d}", beg=0, end=-1) for i in BATCH_SLICE]


def serve_queries(window: int = 100_000, n: int = 10_000) -> List[dict]:
    """Serving stream: 3-5-edge patterns on 2-4 nodes over the 7.8M- and
    63M-edge graphs, delta log-uniform in [600, 604800], 20% enumerations
    with a cap log-uniform in [1e4, 1e6]."""
    graphs = [(synth.SPECS[k].name, synth.SPECS[k].num_edges) for k in ("bursty-1.1m-7.8m", "bursty-6m-63m")]
    return mixed_queries(n, 5, (3, 5), (2, 4), graphs, window, delta_range=(600, 604800), enum_frac=0.2)


# 16 count queries of the serving stream (3-, 4- and 5-edge patterns on both
# graphs, over their 100k-root windows) whose search is cheap (under 2 ms
# each for this library on a B200).
SERVE_SLICE = (4, 5, 7, 11, 24, 3, 13, 14, 17, 18, 1, 6, 8, 10, 12, 16)


def refgen_serve_slice() -> List[dict]:
    """SERVE_SLICE of the serving stream: the slice the reference's
    generated kernel checks."""
    qs = serve_queries(100_000, 10_000)
    return [dict(qs[i], name=f"serve-{i:04d}") for i in SERVE_SLICE]


CONSTRAINED_DELTA = 86400


def constrained_queries() -> List[Tuple[str, List[int], List[int], dict]]:
    """The reference's additional-features query shapes
    (system/queries/additional-features/*-M4-{no,v,t,all,f}.yaml) as
    (name, mu, mv, constraints) on the 7.8M-edge graph with node and edge
    features uniform in [0, 1e9): the reference's delta 3600 and gaps
    900 / 1800 are scaled by 24 (delta 86400).  The "-f" filter names e0, e1,
    e3: the reference's own names the anti-edge e2, which it reads past its
    arrays."""
    m4, m4a = ([0, 1, 2, 3], [1, 2, 3, 0]), ([0, 1, 2, 2, 3], [1, 2, 0, 3, 0])
    nodes = {"node0": "f > 500000000", "node1": "f < 500000000", "node2": "f > 500000000",
             "node3": "f < 500000000"}
    anti = {"antiEdge": [False, False, True, False, False], "temporal": [21600, 43200, 43200, 21600]}
    d = {"delta": CONSTRAINED_DELTA}
    return [("M4-no", *m4, dict(d)), ("M4-v", *m4, dict(d, **nodes)),
            ("M4-t", *m4, dict(d, temporal=[21600, 43200, 21600], **nodes)),
            ("M4-all", *m4a, dict(d, **nodes, **anti)),
            ("M4-f", *m4a, dict(d, filter="(e0 + e1 + e3) > 1000000000", **nodes, **anti))]


def constrained_features(num_vertices: int, num_edges: int, seed: int = 5):
    """Node features per input vertex id and edge features per sorted edge,
    uniform in [0, 1e9)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return (rng.integers(0, 10**9, num_vertices).astype(np.int32),
            rng.integers(0, 10**9, num_edges).astype(np.int32))
