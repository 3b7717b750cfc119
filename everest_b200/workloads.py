"""Named benchmark workloads (synthetic stand-ins for the reference's
SNAP / ethereum graphs, which are not available offline).

Each workload is a graph from ``synth.SPECS`` plus a list of queries
(relabeled motif edges, delta, count or enumerate cap)."""
from __future__ import annotations

from typing import Dict, List

from . import synth

WORKLOADS: Dict[str, dict] = {
    # 10k nodes / 200k edges, triangle 0->1->2->0, delta 3600, count
    "zipf-200k-triangle": {"graph": "zipf-10k-200k", "kind": "triangle", "delta": 3600},
    # 1.1M nodes / 7.8M edges, every connected 3-edge pattern on 2-3 nodes
    # (36 by rule), each run separately, delta 86400, count
    "bursty-7.8m-3edge": {"graph": "bursty-1.1m-7.8m", "kind": "three_edge", "delta": 86400},
}


def queries(name: str) -> List[dict]:
    wl = WORKLOADS[name]
    if wl["kind"] == "triangle":
        return [{"name": "triangle", "mu": [0, 1, 2], "mv": [1, 2, 0], "delta": wl["delta"]}]
    if wl["kind"] == "three_edge":
        out = []
        for i, p in enumerate(synth.three_edge_patterns()):
            out.append({"name": f"3e-{i:02d}", "mu": [a for a, b in p], "mv": [b for a, b in p],
                        "delta": wl["delta"]})
        return out
    raise KeyError(name)
