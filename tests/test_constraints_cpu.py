"""Constraint features on the CPU: the expression compiler against C's own
arithmetic, the oracle against the reference's generated code (fixtures),
and the checks that refuse what the reference cannot run."""
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
