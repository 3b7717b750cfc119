"""Generate the golden fixtures in this directory.

The reference ships no test vectors for this path, so the fixtures are
produced by the reference's own code run here: the host build of its legacy
Baseline search body (``plugins/GPUWorkerBaseline.cu:21-206``, compiled by
``oracle/ref_baseline.mk`` into ``oracle/_ref/``).  Every count written below
is computed by that build AND by the C restatement in ``oracle/``; the script
refuses to write a fixture when they disagree.  The reference's motif files
(``inputs/motifs/M*.txt``) are read from the reference tree and stored as
fixture data.

Run from the repository root, in a container that has the reference tree:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from everest_b200 import synth  # noqa: E402

REF = O.reference_root()  # EVX_REFERENCE_ROOT; required (the script refuses to run without it)


def graph_digest(u, v, t) -> str:
    h = hashlib.sha256()
    for a in (u, v, t):
        h.update(np.ascontiguousarray(a, np.int32).tobytes())
    return h.hexdigest()


def small_graphs():
    """Seeded small graphs covering ties, self-loops, parallel edges, hubs."""
    out = {}
    rng = np.random.Generator(np.random.PCG64(20240601))
    specs = [
        ("empty", 0, 3, 10),
        ("one-edge", 1, 2, 10),
        ("tiny-ties", 40, 5, 6),
        ("tiny-loops", 60, 6, 30),
        ("dense-4", 80, 4, 200),
        ("mid-uniform", 2000, 200, 5000),
        ("mid-hub", 3000, 500, 20000),
        ("mid-ties", 2500, 100, 50),
    ]
    for name, E, V, tmax in specs:
        if name == "mid-hub":
            w = np.arange(1, V + 1, dtype=np.float64) ** -1.2
            w /= w.sum()
            u = rng.choice(V, size=E, p=w)
            v = rng.choice(V, size=E, p=w)
        else:
            u = rng.integers(0, V, size=E)
            v = rng.integers(0, V, size=E)
        if name != "tiny-loops":
            same = u == v
            v[same] = (v[same] + 1) % V
        t = np.sort(rng.integers(0, tmax, size=E))
        out[name] = (u.astype(np.int32), v.astype(np.int32), t.astype(np.int32), V)
    # C1-shaped graph at 1/20 scale (zipf 1.5)
    spec = synth.GraphSpec("zipf-2k-10k", "zipf", 2_000, 10_000, seed=11)
    u, v, t = synth.generate(spec)
    out["zipf-2k-10k"] = (u, v, t, 2_000)
    return out


def reference_motifs():
    mdir = os.path.join(REF, "inputs", "motifs")
    res = {}
    for f in sorted(os.listdir(mdir)):
        if f.endswith(".txt"):
            with open(os.path.join(mdir, f)) as fh:
                res[f[:-4]] = fh.read()
    return res


def both(g, mu, mv, delta, roots=None):
    c_or, st = O.count(g, mu, mv, delta, roots=roots)
    c_ref = None
    if len(set(mu) | set(mv)) <= 5 and len(mu) <= 6:
        c_ref = O.ref_baseline_count(g, mu, mv, delta, roots=roots, threads=os.cpu_count() or 1)
        if c_ref != c_or:
            raise SystemExit(f"oracle {c_or} != reference Baseline {c_ref} for {mu},{mv},{delta}")
    return c_or, c_ref, st


def main():
    O.build()
    if O.ref_lib() is None:
        raise SystemExit("reference Baseline host build missing (needs the reference tree)")
    motifs_txt = reference_motifs()
    motifs = {name: O.parse_motif(txt) for name, txt in motifs_txt.items()}
    three = synth.three_edge_patterns()
    rand = synth.random_patterns(12, (4, 5), (2, 4), seed=7)

    graphs = small_graphs()
    np.savez_compressed(os.path.join(HERE, "small_graphs.npz"),
                        **{f"{n}_u": g[0] for n, g in graphs.items()},
                        **{f"{n}_v": g[1] for n, g in graphs.items()},
                        **{f"{n}_t": g[2] for n, g in graphs.items()},
                        **{f"{n}_V": np.array([g[3]]) for n, g in graphs.items()})
    cases = []
    for gname, (u, v, t, V) in graphs.items():
        print(f"graph {gname}", flush=True)
        g = O.Graph(u, v, t, V)
        tspan = int(t.max() - t.min()) if t.size else 0
        deltas = [0, max(1, tspan // 50)]
        if gname not in ("mid-hub", "zipf-2k-10k"):
            deltas.append(max(1, tspan // 5))  # hub graphs: wide windows explode for k = 5
        if u.size <= 80:
            deltas.append(tspan + 1)  # whole-span window only where it stays small
        deltas = sorted(set(deltas))
        pats = [("3e-%d" % i, [a for a, b in p], [b for a, b in p]) for i, p in enumerate(three)]
        pats += [(n, list(m[0]), list(m[1])) for n, m in motifs.items()]
        pats += [("r-%d" % i, [a for a, b in p], [b for a, b in p]) for i, p in enumerate(rand)]
        for pname, mu, mv in pats:
            for d in deltas:
                c, cref, st = both(g, mu, mv, d)
                cases.append({"graph": gname, "motif": pname, "mu": mu, "mv": mv, "delta": d,
                              "count": c, "reference_baseline": cref,
                              "candidates": st["candidates"]})
                if gname == "mid-uniform" and pname in ("M1", "3e-7") and d == deltas[1]:
                    rb, re_ = 100, 900
                    c2, cref2, _ = both(g, mu, mv, d, roots=(rb, re_))
                    cases.append({"graph": gname, "motif": pname, "mu": mu, "mv": mv, "delta": d,
                                  "roots": [rb, re_], "count": c2, "reference_baseline": cref2})
    # enumeration golden rows (sorted edge ids) on two graphs
    enum_cases = []
    for gname in ("tiny-ties", "dense-4", "mid-ties"):
        u, v, t, V = graphs[gname]
        g = O.Graph(u, v, t, V)
        for pname, (mu, mv) in (("M4", motifs["M4"]), ("3e-7", ([0, 0, 0], [1, 2, 1]))):
            d = max(1, int(t.max() - t.min()) // 5) if t.size else 1
            rows, tot = O.enumerate_rows(g, list(mu), list(mv), d, 10 ** 7)
            enum_cases.append({"graph": gname, "motif": pname, "mu": list(mu), "mv": list(mv),
                               "delta": d, "total": tot,
                               "rows": sorted(map(list, rows.tolist()))})
    # full-size CPU-runnable workload (zipf 10k nodes / 200k edges)
    spec = synth.SPECS["zipf-10k-200k"]
    u, v, t = synth.generate(spec)
    g = O.Graph(u, v, t, spec.num_nodes)
    full = {"graph": spec.name, "digest": graph_digest(u, v, t), "patterns": []}
    c, cref, st = both(g, [0, 1, 2], [1, 2, 0], 3600)
    c_strict, _ = O.count(g, [0, 1, 2], [1, 2, 0], 3600, strict_ts=True)
    full["triangle"] = {"mu": [0, 1, 2], "mv": [1, 2, 0], "delta": 3600, "count": c,
                        "reference_baseline": cref, "strict_ts_count": c_strict, "stats": st}
    for i, p in enumerate(three):
        mu, mv = [a for a, b in p], [b for a, b in p]
        c, cref, st = both(g, mu, mv, 3600)
        full["patterns"].append({"motif": "3e-%d" % i, "mu": mu, "mv": mv, "delta": 3600,
                                 "count": c, "reference_baseline": cref})
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump({"source": "reference Baseline body (host build) + oracle, equal on every case",
                   "reference_motifs": motifs_txt, "cases": cases, "enum_cases": enum_cases,
                   "full_zipf": full}, fh, indent=0)
    print(f"wrote {len(cases)} count cases, {len(enum_cases)} enumeration cases")


if __name__ == "__main__":
    if REF is None:
        raise SystemExit("set EVX_REFERENCE_ROOT to the reference checkout")
    main()
