"""The reference's own generated search code, built for the host.

TEST INFRASTRUCTURE ONLY: the constraint fixtures (tests/golden/
make_constraint_golden.py) and the cpu_baseline leg of
``bench.py --mode constrained`` use it, as the checker and as the timed
reference CPU path.  The product never imports it.

The reference renders one CUDA search kernel per query with KernelGen
(system/tmine/KernelGen.py), writing the constraint snippets into its own
template directory first (system/tmine/Query.py:135-160), so it runs on a
scratch copy of the reference's ``system/`` tree.  With warpCentric,
warpBalancing and tailExpansion off each CUDA thread runs one root's
sequential search; that kernel body (everything before the host launcher)
is compiled for the host with gen_shim.h and run over every root by
gen_driver.cc, one OpenMP iteration per root.  Rendering needs the
reference tree, named by EVX_REFERENCE_ROOT; the built libraries under
oracle/_ref/ run without it.
"""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess
import sys
import tempfile
import types
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_kg = None


def reference_root() -> Optional[str]:
    r = os.environ.get("EVX_REFERENCE_ROOT")
    return r if r and os.path.isdir(os.path.join(r, "system", "tmine")) else None


def available() -> bool:
    return reference_root() is not None


def _drop_tmine() -> None:
    """Forget the tmine package and its submodules imported from a scratch copy."""
    for name in [m for m in sys.modules if m == "tmine" or m.startswith("tmine.")]:
        del sys.modules[name]


def _kernelgen():
    """KernelGen and Query from a scratch copy of the reference's system/."""
    global _kg
    if _kg is None:
        scratch = tempfile.mkdtemp(prefix="evx-kernelgen-")
        ref = reference_root()
        if ref is None:
            raise RuntimeError("set EVX_REFERENCE_ROOT to a reference checkout")
        shutil.copytree(os.path.join(ref, "system"), os.path.join(scratch, "system"))
        pkg = types.ModuleType("tmine")
        pkg.__path__ = [os.path.join(scratch, "system", "tmine")]
        _drop_tmine()  # submodules another scratch copy left behind
        sys.modules["tmine"] = pkg  # bypass tmine/__init__ (it imports the compiled corelib)
        from tmine import KernelGen as KG, Query as Q  # noqa: E402
        _kg = (KG, Q, scratch)
    return _kg


def cleanup() -> None:
    """Remove the scratch copy of the reference's system/ tree."""
    global _kg
    if _kg is not None:
        shutil.rmtree(_kg[2], ignore_errors=True)
        _drop_tmine()
        _kg = None


def render(mu, mv, cons: dict, enum_cap: int = 0) -> str:
    """The generated kernel body for one query (no includes, no launcher)."""
    KG, Q, scratch = _kernelgen()
    motif = os.path.join(scratch, "motif.txt")
    with open(motif, "w") as f:
        for i, (a, b) in enumerate(zip(mu, mv)):
            f.write(f"{a + 1} {b + 1} {i + 1}\n")
    opts = {"gpu": 1, "warpCentric": False, "warpBalancing": False, "tailExpansion": False}
    if enum_cap:
        opts["enumerate"] = enum_cap
    q = Q.Query.__new__(Q.Query)
    q.queryFile = {"pattern": motif, "graph": "-", "constraints": cons, "options": opts}
    q.name = "query"
    q.cons = Q.Constraints(cons)
    o = Q.Options()
    o.update(Q.Options(opts))
    q.opts = o
    q.cons.genConsTemplates()
    src = KG.KernelGen(motif, q).generate()
    body = []
    for line in src.split("\n"):
        if line.startswith("// -----"):
            break
        if line.lstrip().startswith("#include"):
            continue
        body.append(line)
    return "\n".join(body) + "\n"


def compile_body(body: str, out_so: str, enum: bool = False) -> str:
    os.makedirs(os.path.dirname(out_so), exist_ok=True)
    inc = out_so[: -3] + ".inc"
    with open(inc, "w") as f:
        f.write(body)
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-w", "-fpermissive", "-fopenmp",
                    f"-I{HERE}", f'-DGEN_BODY="{inc}"'] + (["-DGEN_ENUM"] if enum else []) +
                   ["-o", out_so, os.path.join(HERE, "gen_driver.cc")], check=True)
    return out_so


class GeneratedSearch:
    """One compiled query: gen_count(...) over roots [0, work)."""

    def __init__(self, so: str):
        self.lib = ctypes.CDLL(so)
        ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        self.lib.gen_count.argtypes = [ip, ctypes.c_int, ip, ip, ip, ip, ip, ip, ip, ip, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ip, ip, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_ulonglong)]
        self.lib.gen_count.restype = ctypes.c_int

    def run(self, g, node_feat, edge_feat, mu, mv, delta: int, rows: Optional[np.ndarray] = None,
            threads: int = 0) -> int:
        """g: an oracle.Graph; node_feat per vertex id, edge_feat per edge."""
        k = len(mu)
        eg = np.stack([g.u, g.v, g.t], axis=1).astype(np.int32).ravel()
        out = ctypes.c_ulonglong(0)
        self.lib.gen_count(eg, g.E, g.in_eid, g.in_off, g.out_eid, g.out_off,
                           np.ascontiguousarray(node_feat, np.int32), np.ascontiguousarray(edge_feat, np.int32),
                           np.asarray(mu, np.int32), np.asarray(mv, np.int32), k, int(delta),
                           max(0, g.E - k + 1), rows if rows is not None else np.zeros(1, np.int32),
                           np.arange(max(g.E, 1), dtype=np.int32), int(threads), ctypes.byref(out))
        return int(out.value)


def bench_library(name: str) -> str:
    return os.path.join(REF_DIR, f"gen_{name}.so")


def build_bench_queries() -> None:
    """Build the reference's search for each constrained bench query into
    oracle/_ref/gen_<name>.so (run where the reference tree exists)."""
    sys.path.insert(0, os.path.dirname(HERE))
    from everest_b200 import workloads
    try:
        for name, mu, mv, cons in workloads.constrained_queries():
            compile_body(render(mu, mv, cons), bench_library(name))
    finally:
        cleanup()
