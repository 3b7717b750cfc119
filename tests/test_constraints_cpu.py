"""Constraint features on the CPU: the expression compiler against C's own
arithmetic, the oracle against the reference's generated code (fixtures),
and the checks that refuse what the reference cannot run."""
import ctypes
import json
import os
import random
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from everest_b200 import consexpr
from everest_b200.constraints import ConstraintError, Constraints, EvxProgram
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _golden():
    with open(os.path.join(GOLD, "constraint_golden.json")) as f:
        return json.load(f)


def _graphs():
    d = np.load(os.path.join(GOLD, "small_graphs.npz"))
    f = np.load(os.path.join(GOLD, "constraint_features.npz"))
    out = {}
    for name in {c["graph"] for c in _golden()["cases"]}:
        g = O.Graph(d[name + "_u"], d[name + "_v"], d[name + "_t"], int(d[name + "_V"][0]))
        out[name] = (g, f[name + "_node"], f[name + "_edge"])
    return out


def test_oracle_matches_reference_generated_code():
    gs = _graphs()
    cases = _golden()["cases"]
    assert len(cases) >= 300
    for c in cases:
        g, nf, ef = gs[c["graph"]]
        cons = Constraints.from_yaml(c["constraints"], c["mu"], c["mv"]).to_struct()
        got = O.count_constrained(g, c["mu"], c["mv"], c["delta"], cons, nf, ef)
        assert got == c["count"], c


def test_unconstrained_struct_equals_plain_search():
    d = np.load(os.path.join(GOLD, "small_graphs.npz"))
    g = O.Graph(d["mid-hub_u"], d["mid-hub_v"], d["mid-hub_t"], int(d["mid-hub_V"][0]))
    for mu, mv in (([0, 1, 2], [1, 2, 0]), ([0, 1, 2, 3], [1, 2, 3, 0]), ([0, 0, 1], [1, 2, 2])):
        cons = Constraints.from_yaml({"delta": 1000}, mu, mv)
        assert cons.empty
        assert O.count_constrained(g, mu, mv, 1000, cons.to_struct()) == O.count(g, mu, mv, 1000)[0]


def _rand_expr(rng, depth, names):
    if depth == 0 or rng.random() < 0.25:
        r = rng.random()
        if r < 0.45:
            return rng.choice(names)
        if r < 0.9:
            return str(rng.choice([0, 1, 2, 3, 7, 10, 255, 65536, 2147483647, 1000000007]))
        return str(rng.choice([4294967296, 9000000000000]))  # long literals
    op = rng.choice(["+", "-", "*", "/", "%", "<<", ">>", "<", "<=", ">", ">=", "==", "!=",
                     "&", "^", "|", "&&", "||", "u-", "u!", "u~", "?"])
    if op.startswith("u"):
        return f"{op[1]}({_rand_expr(rng, depth - 1, names)})"
    if op == "?":
        return (f"({_rand_expr(rng, depth - 1, names)}) ? ({_rand_expr(rng, depth - 1, names)}) : "
                f"({_rand_expr(rng, depth - 1, names)})")
    a, b = _rand_expr(rng, depth - 1, names), _rand_expr(rng, depth - 1, names)
    if op in ("/", "%"):
        b = f"(({b}) | 1)"  # C leaves division by zero undefined
        a = f"(({a}) & 0x3fffffff)"  # and INT_MIN / -1
    if op in ("<<", ">>"):
        b = f"(({b}) & 15)"  # and shifts past the width
        if op == "<<":
            a = f"(({a}) & 0xffff)"  # and left shifts of negative values
    return f"({a}) {op} ({b})"


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_compiler_matches_c_arithmetic():
    """Each program, run by the host interpreter and by the oracle's, gives
    what gcc's own evaluation of the same C expression gives."""
    rng = random.Random(7)
    names = ["e0", "e1", "e2"]
    exprs = [_rand_expr(rng, 3, names) for _ in range(400)]
    values = [(0, 0, 0), (1, -1, 7), (2147483647, -2147483648, 3), (123456, -99, 65535),
              (-5, 9, 1000000000)]
    src = ["#include <stdio.h>", "int main(void) {"]
    for vals in values:
        src.append("{ int e0 = %d, e1 = %d, e2 = %d;" % vals)
        for e in exprs:
            src.append('  printf("%%lld\\n", (long long)(%s));' % e)
        src.append("}")
    src.append("return 0; }")
    with tempfile.TemporaryDirectory() as tmp:
        c = os.path.join(tmp, "x.c")
        with open(c, "w") as f:
            f.write("\n".join(src))
        exe = os.path.join(tmp, "x")
        subprocess.run(["gcc", "-O0", "-fwrapv", "-w", "-o", exe, c], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    i = 0
    for vals in values:
        for e in exprs:
            code = consexpr.compile_expr(e, "e", num_edges=3)
            p = EvxProgram()
            p.len = len(code)
            for j, (op, arg) in enumerate(code):
                p.op[j], p.arg[j] = op, arg
            want = int(out[i])
            assert consexpr.evaluate(code, vals) == want, (e, vals)
            assert O.prog_eval(p, vals) == want, (e, vals)
            i += 1


def test_expression_errors():
    for bad in ("f >", "g > 1", "f > 1u", "f > 0xffffffff", "(f", "f > 1 2", "e0 > 1"):
        with pytest.raises(consexpr.ExprError):
            consexpr.compile_expr(bad, "f")
    with pytest.raises(consexpr.ExprError):
        consexpr.compile_expr("e3 > 1", "e", num_edges=3)
    with pytest.raises(consexpr.ExprError):
        consexpr.compile_expr("e1 > 1", "e", num_edges=3, allowed_edges=[0, 2])
    assert consexpr.evaluate(consexpr.compile_expr("f > 500000000", "f"), [500000001]) == 1
    # int arithmetic wraps; a long literal widens it
    assert consexpr.evaluate(consexpr.compile_expr("e0 + e1", "e", num_edges=2), [2**31 - 1, 1]) == -2**31
    assert consexpr.evaluate(consexpr.compile_expr("e0 + e1 + 0L", "e", num_edges=2), [2**31 - 1, 1]) == -2**31
    assert consexpr.evaluate(consexpr.compile_expr("0L + e0 + e1", "e", num_edges=2), [2**31 - 1, 1]) == 2**31


def test_constraint_checks():
    m4a = ([0, 1, 2, 2, 3], [1, 2, 0, 3, 0])
    ok = Constraints.from_yaml({"delta": 3600, "antiEdge": [False, False, True, False, False],
                                "temporal": [900, 1800, 1800, 900], "node0": "f > 5", "node1": "f < 5",
                                "node2": "f > 5", "node3": "f < 5", "filter": "e0 + e1 + e3 > 10"}, *m4a)
    s = ok.to_struct()
    assert s.anti_mask == 4 and s.has_temporal == 1 and s.node_mode == 2 and s.has_filter == 1
    bad = [
        ({"antiEdge": [False, True, False, False, False]}, "motif edge 1"),
        ({"antiEdge": [False, False, False, False, True]}, "motif edge 4"),
        ({"antiEdge": [True, False, False, False, False]}, "motif edge 0"),
        ({"antiEdge": [False, False]}, "entries"),
        ({"antiEdge": [False, False, True, False, False], "filter": "e2 > 1"}, "not a matched edge"),
        ({"temporal": [1, 2]}, "needs 4"),
        ({"node0": "f > 1", "node1": "f > 1"}, "motif with 4 nodes"),
        ({"node0": "f > 1", "node2": "f > 1", "node3": "f", "node4": "f"}, "without gaps"),
        ({"node": "f > 1", "node0": "f > 1"}, "not both"),
        ({"edge0": "f > 1", "edge1": "f > 1"}, "per-edge"),
        ({"label": 3}, "unsupported"),
    ]
    for cons, msg in bad:
        with pytest.raises((ConstraintError, consexpr.ExprError), match=msg):
            Constraints.from_yaml(dict(cons, delta=3600), *m4a)
    # entries as the reference renders them into C++: true / false / 1 / 0, any case
    st = Constraints.from_yaml({"delta": 1, "antiEdge": ["False", 0, "TRUE", False, "false"]}, *m4a).to_struct()
    assert st.anti_mask == 4
    with pytest.raises(ConstraintError, match="not a boolean"):
        Constraints.from_yaml({"delta": 1, "antiEdge": [False, False, "yes", False, False]}, *m4a)
    # an anti-edge must join nodes that earlier real edges map
    with pytest.raises(ConstraintError, match="no earlier real edge"):
        Constraints.from_yaml({"delta": 1, "antiEdge": [False, False, True, False]},
                              [0, 1, 1, 2], [1, 2, 3, 0])


def test_oracle_rows_match_reference_generated_enumeration():
    """The generated enumeration body's rows (Euid of e_0 .. e_{k-1}, here
    the sorted edge ids) equal the oracle's, as multisets."""
    gs = _graphs()
    cases = _golden()["enum_cases"]
    assert len(cases) >= 8
    for c in cases:
        g, nf, ef = gs[c["graph"]]
        cons = Constraints.from_yaml(c["constraints"], c["mu"], c["mv"]).to_struct()
        rows, total = O.enumerate_constrained(g, c["mu"], c["mv"], c["delta"], cons, c["total"] + 5, nf, ef)
        assert total == c["total"]
        assert sorted(map(tuple, rows.tolist())) == [tuple(r) for r in c["rows"]], c["motif"]


def _brute(u, v, t, mu, mv, delta, anti, gaps, node_ok, edge_ok, filt, ef):
    """Direct restatement of the documented semantics over all increasing
    tuples of real edges (tiny graphs only)."""
    import itertools
    k, E = len(mu), len(u)
    real = [j for j in range(k) if not anti[j]]
    prev = {}
    for j in range(1, k):
        p = j - 1
        while p > 0 and anti[p]:
            p -= 1
        prev[j] = p

    def window(j, e):  # e: motif edge -> edge id of the real ones
        t0 = t[e[0]]
        if gaps is None:
            return t0 + delta
        w = t[e[prev[j]]] + gaps[j - 1]
        return w if j == 1 else min(w, t0 + delta)

    total = 0
    for tup in itertools.combinations(range(E), len(real)):
        e = dict(zip(real, tup))
        if u[e[0]] == v[e[0]]:
            continue
        phi, ok = {}, True
        for j in real:
            for a, x in ((mu[j], u[e[j]]), (mv[j], v[e[j]])):
                if phi.setdefault(a, x) != x:
                    ok = False
        if not ok or len(set(phi.values())) != len(phi):
            continue
        if not all(node_ok(a, x) for a, x in phi.items()) or not all(edge_ok(e[j]) for j in real):
            continue
        if not all(t[e[j]] <= window(j, e) for j in real if j > 0):
            continue
        dead = False
        for j in range(1, k):
            if anti[j]:
                tl = window(j, e)
                if any(x > e[prev[j]] and t[x] <= tl and u[x] == phi[mu[j]] and v[x] == phi[mv[j]] and edge_ok(x)
                       for x in range(E)):
                    dead = True
        if dead or (filt is not None and not filt([ef[e[j]] if j in e else 0 for j in range(k)])):
            continue
        total += 1
    return total


def test_oracle_matches_brute_force_semantics():
    """The semantics written in include/everest_b200.h, restated as a
    brute-force check, give the oracle's counts on random tiny graphs."""
    rng = np.random.Generator(np.random.PCG64(99))
    motifs = [([0, 1, 2], [1, 2, 0], [False] * 3), ([0, 1, 0], [1, 0, 1], [False] * 3),
              ([0, 1, 2, 2, 3], [1, 2, 0, 3, 0], [False, False, True, False, False]),
              ([0, 1, 1, 0, 2], [1, 2, 0, 2, 0], [False, False, True, False, False]),
              ([0, 1, 2, 1, 2, 3], [1, 2, 0, 0, 3, 0], [False, False, True, True, False, False]),
              ([0, 1], [1, 2], [False, False]), ([0, 0, 1], [1, 2, 2], [False] * 3)]
    checked = 0
    for trial in range(200):
        E, V = int(rng.integers(8, 22)), int(rng.integers(3, 6))
        u = rng.integers(0, V, E).astype(np.int32)
        v = rng.integers(0, V, E).astype(np.int32)
        t = np.sort(rng.integers(0, 12, E)).astype(np.int32)
        nf = rng.integers(0, 4, V).astype(np.int32)
        ef = rng.integers(0, 4, E).astype(np.int32)
        mu, mv, anti = motifs[trial % len(motifs)]
        k, n = len(mu), max(max(mu), max(mv)) + 1
        delta = int(rng.integers(2, 10))
        cons = {"delta": delta}
        if any(anti):
            cons["antiEdge"] = anti
        gaps = None
        if trial % 2:
            gaps = [int(x) for x in rng.integers(0, 12, k - 1)]
            cons["temporal"] = gaps
        th = [int(x) for x in rng.integers(0, 3, n)]
        if trial % 3 == 0:
            cons.update({f"node{a}": f"f >= {th[a]}" for a in range(n)})
        if trial % 4 == 1:
            cons["edge"] = "f != 2"
        real = [j for j in range(k) if not anti[j]]
        filt = None
        if trial % 5 == 2:
            cons["filter"] = " + ".join(f"e{j}" for j in real) + f" > {len(real)}"
            filt = lambda vals: sum(vals[j] for j in real) > len(real)  # noqa: E731
        node_ok = (lambda a, x: nf[x] >= th[a]) if trial % 3 == 0 else (lambda a, x: True)
        edge_ok = (lambda x: ef[x] != 2) if trial % 4 == 1 else (lambda x: True)
        want = _brute(u, v, t, mu, mv, delta, anti, gaps, node_ok, edge_ok, filt, ef)
        g = O.Graph(u, v, t, V)
        c = Constraints.from_yaml(cons, mu, mv).to_struct()
        roots = (0, max(0, E - k + 1))
        got = O.count_constrained(g, mu, mv, delta, c, nf, ef, roots=roots)
        assert got == want, (trial, cons, got, want)
        checked += want > 0
    assert checked > 40


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_struct_layout_matches_the_c_header():
    """The ctypes mirror of evx_constraints / evx_program has the C layout."""
    from everest_b200.constraints import EvxConstraints
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    fields = ["anti_mask", "has_temporal", "temporal", "node_mode", "node", "has_edge", "edge", "has_filter",
              "filter"]
    src = ["#include <stdio.h>", "#include <stddef.h>", '#include "everest_b200.h"', "int main(void) {",
           '  printf("%zu %zu\\n", sizeof(evx_constraints), sizeof(evx_program));']
    src += [f'  printf("%zu\\n", offsetof(evx_constraints, {f}));' for f in fields]
    src += ["  return 0; }"]
    with tempfile.TemporaryDirectory() as tmp:
        c = os.path.join(tmp, "x.c")
        with open(c, "w") as f:
            f.write("\n".join(src))
        exe = os.path.join(tmp, "x")
        subprocess.run(["gcc", "-I", os.path.join(root, "include"), "-o", exe, c], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    assert int(out[0]) == ctypes.sizeof(EvxConstraints) and int(out[1]) == ctypes.sizeof(EvxProgram)
    for f, off in zip(fields, out[2:]):
        assert getattr(EvxConstraints, f).offset == int(off), f
