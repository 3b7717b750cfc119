"""YAML query model (the reference's system/tmine/Query.py:6-37,311-338).

    pattern: M3.txt            # motif file (u v t lines)
    graph: wiki-talk.txt       # temporal edge list (u v t lines)
    constraints:
      delta: 86400
      node0: f > 500000000     # optional: node predicates (or `node` for all)
      edge: f % 2 == 0         # optional: edge predicate
      temporal: [900, 1800]    # optional: gap bound of each edge after the previous one
      antiEdge: [False, False, True, False, False]   # optional: edges that must not exist
      filter: (e0 + e1) > 100  # optional: over the matched edges' features
    options:
      gpu: 1
      enumerate: 1000          # optional: enumerate up to this many rows
      warpCentric: True        # accepted; the kernels are always warp-centric
      warpBalancing: True      # False disables work stealing
      tailExpansion: True      # False disables range-arithmetic tail counting

The constraints are checked against the motif when the query runs
(everest_b200.constraints.Constraints.from_yaml, which refuses what the
reference's generated code cannot run); node and edge predicates and filters
read the features of the random-feature file (EVX_RAND_FILE).
"""
import os

import yaml

from . import locations

DEFAULT_OPTIONS = {"gpu": 1, "warpCentric": True, "warpBalancing": True, "tailExpansion": True}


class Options:
    def __init__(self, opts=None):
        self.opts = dict(DEFAULT_OPTIONS)
        if opts:
            self.opts.update(opts)
        if self.multigpu():
            self.opts["multigpu"] = True

    def gpu(self) -> int:
        return int(self.opts["gpu"])

    def multigpu(self) -> bool:
        return int(self.opts["gpu"]) > 1

    def enumerate(self) -> bool:
        return "enumerate" in self.opts

    def enumNum(self) -> int:
        return int(self.opts["enumerate"])

    def flags(self) -> int:
        """EVX_FLAG_* bits the options select."""
        f = 0
        if not self.opts.get("warpBalancing", True):
            f |= 4
        if not self.opts.get("tailExpansion", True):
            f |= 8
        if self.opts.get("strictTimestamps", False):
            f |= 1
        return f

    def __repr__(self):
        return f"Options:\n {self.opts}"


class Constraints:
    def __init__(self, cons):
        self.cons = dict(cons or {})
        if "delta" not in self.cons:
            raise ValueError("query constraints need 'delta'")

    def isTemporal(self) -> bool:
        return "temporal" in self.cons

    def isAnti(self) -> bool:
        return "antiEdge" in self.cons

    def isFilter(self) -> bool:
        return "filter" in self.cons

    def compile(self, mu, mv):
        """The checked, compiled constraints for a motif (relabeled edges)."""
        from ..constraints import Constraints as Compiled
        return Compiled.from_yaml(self.cons, mu, mv)

    def isDelta(self) -> bool:
        return "delta" in self.cons

    def delta(self) -> int:
        return int(self.cons["delta"])

    def genConsTemplates(self):
        """No code generation on this path (kept for call compatibility)."""
        return None

    def __repr__(self):
        return f"Constraints:\n {self.cons}"


def _resolve(name: str, root: str, base_dir: str) -> str:
    if os.path.isabs(name) and os.path.exists(name):
        return name
    for cand in (os.path.join(root, name), os.path.join(base_dir, name)):
        if os.path.exists(cand):
            return cand
    return os.path.join(root, name)


class Query:
    def __init__(self, pathToQuery: str):
        with open(pathToQuery) as f:
            self.queryFile = yaml.safe_load(f)
        self.name = pathToQuery
        base = os.path.dirname(os.path.abspath(pathToQuery))
        for key in ("pattern", "graph", "constraints"):
            if key not in self.queryFile:
                raise ValueError(f"query {pathToQuery} has no '{key}'")
        self.cons = Constraints(self.queryFile["constraints"])
        self.opts = Options(self.queryFile.get("options") or {})
        self.queryFile["pattern"] = _resolve(str(self.queryFile["pattern"]), locations.inputMotifsRoot(), base)
        self.queryFile["graph"] = _resolve(str(self.queryFile["graph"]), locations.inputGraphRoot(), base)

    def pattern(self) -> str:
        return self.queryFile["pattern"]

    def graph(self) -> str:
        return self.queryFile["graph"]

    def constraints(self) -> Constraints:
        return self.cons

    def options(self) -> Options:
        return self.opts

    def __repr__(self):
        return f"Query {self.name}:\n {self.queryFile}"
