"""Algorithmic-work figures of the benchmark workloads (the serial reference
semantics, counted by the instrumented oracle): per query the match count,
roots, CSR offset-pair reads, list openings and candidates examined, from
which bytes_alg = 12 roots + 8 r_reads + 16 candidates.

bench.py reads the JSON this writes (it never runs the oracle outside its
cpu_baseline leg).  Run from the repository root (named workloads only, the
others kept as they are in the JSON; all when none is named):
    python tests/golden/make_workload_stats.py [workload ...]
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from everest_b200 import synth, workloads  # noqa: E402


def main(names):
    path = os.path.join(HERE, "workload_stats.json")
    out = {}
    if names and os.path.exists(path):
        with open(path) as f:
            out = json.load(f)
    for wname, wl in workloads.WORKLOADS.items():
        if not wl.get("stats", True) or (names and wname not in names):
            continue
        spec = synth.SPECS[wl["graph"]]
        u, v, t = synth.load_or_generate(spec.name)
        g = O.Graph(u, v, t, spec.num_nodes)
        rows = []
        for q in workloads.queries(wname):
            c, st = O.count(g, q["mu"], q["mv"], q["delta"], threads=os.cpu_count() or 1)
            st["bytes_alg"] = 12 * st["roots"] + 8 * st["r_reads"] + 16 * st["candidates"]
            rows.append({"name": q["name"], "mu": q["mu"], "mv": q["mv"], "delta": q["delta"],
                         "count": c, **st})
            print(wname, q["name"], c, flush=True)
        out[wname] = {"graph": spec.name, "queries": rows}
    with open(path, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:])
