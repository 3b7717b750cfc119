"""Write constraint_golden.json: constrained counts computed by the
reference's OWN generated search code, checked against the oracle.

For every case the reference's KernelGen renders the per-query CUDA search
with warpCentric, warpBalancing and tailExpansion off, so one CUDA thread runs
one root's sequential search; oracle/ref_generated.py compiles that kernel
body for the host (oracle/gen_shim.h, oracle/gen_driver.cc) and runs it over
every root.  The oracle (oracle/evx_oracle_cons.c) must agree on every case,
or nothing is written.

Needs the reference tree (named by EVX_REFERENCE_ROOT),
g++ and PyYAML; run it where those exist:

    python tests/golden/make_constraint_golden.py
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from everest_b200.constraints import Constraints  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import ref_generated as RG  # noqa: E402

GRAPHS = {"tiny-ties": 2, "dense-4": 20, "mid-ties": 5, "mid-uniform": 250, "mid-hub": 1000,
          "zipf-2k-10k": 200000}
MOTIFS = {
    "path2": ([0, 1], [1, 2]),
    "pair2": ([0, 1], [1, 0]),
    "tri": ([0, 1, 2], [1, 2, 0]),
    "star3": ([0, 0, 0], [1, 2, 3]),
    "rep3": ([0, 1, 0], [1, 0, 1]),
    "M4": ([0, 1, 2, 3], [1, 2, 3, 0]),
    "M4-A": ([0, 1, 2, 2, 3], [1, 2, 0, 3, 0]),
    "anti2": ([0, 1, 2, 1, 2, 3], [1, 2, 0, 0, 3, 0]),
    "anti-fan": ([0, 1, 1, 0, 2], [1, 2, 0, 2, 0]),
}
ANTI = {"M4-A": [False, False, True, False, False],
        "anti2": [False, False, True, True, False, False],
        "anti-fan": [False, False, True, False, False]}
ENUM_CAP = 50_000
ENUM_CASES = [
    ("dense-4", "tri", {"node": "f > 3"}),
    ("mid-hub", "tri", {"node": "f > 3"}),
    ("mid-hub", "rep3", {"temporal": [500, 300], "edge": "f % 3 != 1"}),
    ("mid-hub", "M4", {"node0": "f % 2 == 0", "node1": "f < 7", "node2": "f != 3", "node3": "f >= 2"}),
    ("mid-hub", "tri", {"node": "f > 2", "temporal": [600, 300], "filter": "e0 * e1 > 10"}),
    ("mid-ties", "star3", {"node": "f > 3"}),
    ("zipf-2k-10k", "star3", {"node": "f > 2", "temporal": [120000, 60000], "filter": "e0 * e1 > 10"}),
    ("mid-uniform", "star3", {"filter": "e0 + e1 > 9"}),
]
PER_NODE = ["f % 2 == 0", "f < 7", "f != 3", "f >= 2", "(f & 1) || f > 5"]


def constraint_sets(name, k, n, delta):
    real = [j for j in range(k) if not ANTI.get(name, [False] * k)[j]]
    gaps = [max(1, delta // (2 + (j % 3))) for j in range(k - 1)]
    wide = [delta * 2] + [delta] * (k - 2)
    filt = " + ".join(f"e{j}" for j in real if j < k - 1) + f" > {4 * max(1, len(real) - 1)}"
    out = []
    base = {"delta": delta}
    if name in ANTI:
        out.append(dict(base, antiEdge=ANTI[name]))
        out.append(dict(base, antiEdge=ANTI[name], temporal=gaps))
        out.append(dict(base, antiEdge=ANTI[name], node="f > 2", edge="f % 3 != 1"))
        out.append(dict(base, antiEdge=ANTI[name], filter=filt,
                        **{f"node{a}": PER_NODE[a % len(PER_NODE)] for a in range(n)}))
        return out
    out.append(dict(base, node="f > 4"))
    out.append(dict(base, **{f"node{a}": PER_NODE[a % len(PER_NODE)] for a in range(n)}))
    out.append(dict(base, edge="f % 3 != 1"))
    out.append(dict(base, temporal=gaps))
    out.append(dict(base, temporal=wide))
    out.append(dict(base, filter=filt))
    out.append(dict(base, node="-f < -1 && f * 3 <= 24", edge="(f ^ 5) > 2", temporal=gaps, filter=filt))
    return out


def build(scratch, mu, mv, cons, tag, enum_cap=0):
    so = os.path.join(scratch, f"gen_{tag}.so")
    return RG.GeneratedSearch(RG.compile_body(RG.render(mu, mv, cons, enum_cap), so, enum=enum_cap > 0))


def main():
    d = np.load(os.path.join(HERE, "small_graphs.npz"))
    rng = np.random.Generator(np.random.PCG64(20261203))
    feats = {}
    cases = []
    with tempfile.TemporaryDirectory() as scratch:
        tag = 0
        for gname, delta in GRAPHS.items():
            g = O.Graph(d[gname + "_u"], d[gname + "_v"], d[gname + "_t"], int(d[gname + "_V"][0]))
            nf = rng.integers(0, 10, g.V).astype(np.int32)
            ef = rng.integers(0, 10, max(g.E, 1)).astype(np.int32)
            feats[gname + "_node"], feats[gname + "_edge"] = nf, ef
            for mname, (mu, mv) in MOTIFS.items():
                k, n = len(mu), max(max(mu), max(mv)) + 1
                for cons in constraint_sets(mname, k, n, delta):
                    ref = build(scratch, mu, mv, cons, tag).run(g, nf, ef, mu, mv, delta)
                    tag += 1
                    c = Constraints.from_yaml(cons, mu, mv).to_struct()
                    mine = O.count_constrained(g, mu, mv, delta, c, nf, ef)
                    if mine != ref:
                        raise SystemExit(f"oracle {mine} != reference {ref}: {gname} {mname} {cons}")
                    cases.append({"graph": gname, "motif": mname, "mu": mu, "mv": mv, "delta": delta,
                                  "constraints": cons, "count": ref})
                    print(f"{gname:12s} {mname:8s} {ref:10d} {sorted(k for k in cons if k != 'delta')}")
        # enumeration: the generated enumeration body's rows (Euid = sorted
        # edge id here) against the oracle's, every total under the cap
        enum_cases = []
        for gname, mname, cons in ENUM_CASES:
            g = O.Graph(d[gname + "_u"], d[gname + "_v"], d[gname + "_t"], int(d[gname + "_V"][0]))
            nf, ef = feats[gname + "_node"], feats[gname + "_edge"]
            mu, mv = MOTIFS[mname]
            k = len(mu)
            cons = dict(cons, delta=GRAPHS[gname])
            rows = np.zeros(ENUM_CAP * k, np.int32)
            total = build(scratch, mu, mv, cons, tag, ENUM_CAP).run(g, nf, ef, mu, mv, GRAPHS[gname], rows)
            tag += 1
            if not 0 < total < ENUM_CAP:
                raise SystemExit(f"enumeration case {gname} {mname} {cons}: total {total}")
            ref_rows = sorted(map(tuple, rows[: total * k].reshape(total, k).tolist()))
            c = Constraints.from_yaml(cons, mu, mv).to_struct()
            o_rows, o_total = O.enumerate_constrained(g, mu, mv, GRAPHS[gname], c, ENUM_CAP, nf, ef)
            if o_total != total or sorted(map(tuple, o_rows.tolist())) != ref_rows:
                raise SystemExit(f"oracle rows differ from the reference's: {gname} {mname} {cons}")
            enum_cases.append({"graph": gname, "motif": mname, "mu": mu, "mv": mv, "delta": GRAPHS[gname],
                               "constraints": cons, "total": total, "rows": [list(r) for r in ref_rows]})
            print(f"enumerate {gname:12s} {mname:8s} {total:6d} rows")
    RG.cleanup()
    np.savez_compressed(os.path.join(HERE, "constraint_features.npz"), **feats)
    with open(os.path.join(HERE, "constraint_golden.json"), "w") as f:
        json.dump({"source": "reference KernelGen output (warp options off) run on the host; "
                             "oracle/evx_oracle_cons.c agrees on every case",
                   "features": "constraint_features.npz", "cases": cases, "enum_cases": enum_cases},
                  f, indent=0)
    print(len(cases), "cases")


if __name__ == "__main__":
    main()
