"""Query constraints: the reference's YAML `constraints` block as data.

The reference turns each constraint into C code generated per query
(system/tmine/Query.py:39-310, system/tmine/KernelGen.py:288-336,467-534).
Here `Constraints.from_yaml` checks the same keys, compiles the expressions
(everest_b200/consexpr.py) and fills the `evx_constraints` struct of
include/everest_b200.h, which one precompiled kernel reads.

Accepted keys (besides `delta`):
  node                    one predicate in `f` for every motif node
  node0 .. node{n-1}      one per motif node (extra ones are ignored, as in
                          the reference's nodeConstraints[] table)
  edge                    one predicate in `f` for every edge
  temporal                k-1 gap bounds (extra ones are ignored)
  antiEdge                k booleans
  filter                  an expression in e0 .. e{k-1} (the reference's
                          generated code declares eid0 .. eid{k-2} only, so
                          naming the last edge, e{k-1}, is an extension)

Refused, with the reason:
  edge0, edge1, ...       the reference applies edge1's predicate to e_0 and
                          edge0's to every later edge (Query.py:249-301)
  an anti-edge as motif edge 0, 1 or k-1, or one touching a node no earlier
                          real edge maps: the generated search never ends or
                          reads past its arrays there
  a filter naming an anti-edge (it reads the feature of edge id E)
  node0.. fewer than the motif's nodes (nodeConstraints[] is indexed past
                          its end)
"""
from __future__ import annotations

import ctypes
import re
from typing import Optional, Sequence

from . import consexpr

MAX_EDGES = 8
MAX_NODES = 9


class EvxProgram(ctypes.Structure):
    _fields_ = [("len", ctypes.c_int32), ("op", ctypes.c_int32 * consexpr.PROG_MAX),
                ("arg", ctypes.c_int64 * consexpr.PROG_MAX)]


class EvxConstraints(ctypes.Structure):
    _fields_ = [("anti_mask", ctypes.c_uint32), ("has_temporal", ctypes.c_int32),
                ("temporal", ctypes.c_int32 * (MAX_EDGES - 1)), ("node_mode", ctypes.c_int32),
                ("node", EvxProgram * MAX_NODES), ("has_edge", ctypes.c_int32), ("edge", EvxProgram),
                ("has_filter", ctypes.c_int32), ("filter", EvxProgram)]


def _fill(p: EvxProgram, code) -> None:
    p.len = len(code)
    for i, (op, arg) in enumerate(code):
        p.op[i] = op
        p.arg[i] = arg


class ConstraintError(ValueError):
    pass


def _flag(x) -> bool:
    """An antiEdge entry as the reference renders it into C++
    (str(x).lower(), Query.py:44-50): true / false, or 1 / 0."""
    text = str(x).strip().lower()
    if text in ("true", "1"):
        return True
    if text in ("false", "0"):
        return False
    raise ConstraintError(f"antiEdge entry {x!r} is not a boolean")


class Constraints:
    """Validated, compiled constraints of one query on one motif."""

    KEYS = ("delta", "node", "edge", "temporal", "antiEdge", "filter")

    def __init__(self):
        self.anti = []
        self.temporal: Optional[list] = None
        self.node_mode = 0
        self.node_code = []
        self.edge_code = None
        self.filter_code = None
        self.source = {}

    @property
    def empty(self) -> bool:
        return (not any(self.anti) and self.temporal is None and self.node_mode == 0
                and self.edge_code is None and self.filter_code is None)

    @classmethod
    def from_yaml(cls, cons: dict, mu: Sequence[int], mv: Sequence[int]) -> "Constraints":
        k = len(mu)
        n = max(max(mu), max(mv)) + 1
        self = cls()
        self.source = dict(cons)
        node_keys = sorted(key for key in cons if re.fullmatch(r"node\d+", key))
        edge_keys = [key for key in cons if re.fullmatch(r"edge\d+", key)]
        for key in cons:
            if key in cls.KEYS or key in node_keys:
                continue
            if key in edge_keys:
                raise ConstraintError(
                    f"constraint {key!r}: per-edge predicates are not supported (the reference "
                    "applies edge1's predicate to the first edge and edge0's to every later one)")
            raise ConstraintError(f"unsupported constraint {key!r}")
        # anti-edges
        if "antiEdge" in cons:
            anti = [_flag(x) for x in cons["antiEdge"]]
            if len(anti) != k:
                raise ConstraintError(f"antiEdge has {len(anti)} entries for a {k}-edge motif")
            for j in (0, 1, k - 1):
                if anti[j]:
                    raise ConstraintError(f"motif edge {j} cannot be an anti-edge (the reference's "
                                          "search never ends or reads past its arrays there)")
            seen = {mu[0], mv[0]}
            for j in range(1, k):
                if anti[j] and not (mu[j] in seen and mv[j] in seen):
                    raise ConstraintError(f"anti-edge {j} touches a node that no earlier real edge maps")
                if not anti[j]:
                    seen.update((mu[j], mv[j]))
            self.anti = anti
        else:
            self.anti = [False] * k
        # temporal gaps
        if "temporal" in cons:
            tem = [int(x) for x in cons["temporal"]]
            if len(tem) < k - 1:
                raise ConstraintError(f"temporal has {len(tem)} entries; a {k}-edge motif needs {k - 1}")
            self.temporal = tem[:k - 1]
            for g in self.temporal:
                if not -(1 << 31) <= g < (1 << 31):
                    raise ConstraintError("temporal entries must be int32")
        # node predicates
        if "node" in cons and node_keys:
            raise ConstraintError("give either `node` or `node0..`, not both")
        if "node" in cons:
            self.node_mode = 1
            self.node_code = [consexpr.compile_expr(cons["node"], "f")]
        elif node_keys:
            idx = sorted(int(key[4:]) for key in node_keys)
            if idx != list(range(len(idx))):
                raise ConstraintError("node predicates must be node0, node1, ... without gaps")
            if len(idx) < n:
                raise ConstraintError(f"{len(idx)} node predicates for a motif with {n} nodes")
            self.node_mode = 2
            self.node_code = [consexpr.compile_expr(cons[f"node{a}"], "f") for a in range(n)]
        if "edge" in cons:
            self.edge_code = consexpr.compile_expr(cons["edge"], "f")
        if "filter" in cons:
            real = [j for j in range(k) if not self.anti[j]]
            self.filter_code = consexpr.compile_expr(cons["filter"], "e", num_edges=k, allowed_edges=real)
        return self

    def needs_node_features(self) -> bool:
        return self.node_mode != 0

    def needs_edge_features(self) -> bool:
        return self.edge_code is not None or self.filter_code is not None

    def to_struct(self) -> EvxConstraints:
        c = EvxConstraints()
        c.anti_mask = sum(1 << j for j, a in enumerate(self.anti) if a)
        if self.temporal is not None:
            c.has_temporal = 1
            for i, g in enumerate(self.temporal):
                c.temporal[i] = g
        c.node_mode = self.node_mode
        for a, code in enumerate(self.node_code):
            _fill(c.node[a], code)
        if self.edge_code is not None:
            c.has_edge = 1
            _fill(c.edge, self.edge_code)
        if self.filter_code is not None:
            c.has_filter = 1
            _fill(c.filter, self.filter_code)
        return c
