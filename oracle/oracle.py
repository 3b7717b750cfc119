"""Python face of the CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``, and only as
the checker or as the timed CPU baseline.  The product (``everest_b200``)
never imports this module.

* ``liboracle.so`` (``evx_oracle.c``): C restatement of the reference's
  count / enumerate semantics, instrumented for the algorithmic-bytes model.
* ``_ref/gen_<query>.so``: the search the reference generates per query
  (KernelGen, warp options off), built for the host by ``ref_generated.py``
  for the constrained bench queries.
* ``_ref/libref_baseline.so``: the reference's own legacy Baseline search body
  (``plugins/GPUWorkerBaseline.cu:21-206``) compiled for the host by
  ``ref_baseline.mk``; present only where the reference tree was available at
  build time.
* ``parse_motif``: restatement of ``TemporalGraph::ReadGraph`` +
  ``HostMotifData`` (``src/core/cpu/Graph.cc:198-258``,
  ``src/core/cpu/data.cc:411-449``).
* ``brute_force``: direct k-tuple enumeration for graphs of a few dozen edges.
"""
from __future__ import annotations

import ctypes
import itertools
import os
import subprocess
from typing import List, Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libref_baseline.so")
REF_GPU_LIB_PATH = os.path.join(HERE, "_ref", "libref_baseline_gpu.so")

_lib = None
_ref = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


class OracleStats(ctypes.Structure):
    _fields_ = [("roots", ctypes.c_uint64), ("r_reads", ctypes.c_uint64),
                ("candidates", ctypes.c_uint64), ("list_opens", ctypes.c_uint64),
                ("matches", ctypes.c_uint64)]

    def as_dict(self):
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


def reference_root() -> Optional[str]:
    """The reference checkout named by EVX_REFERENCE_ROOT, or None when the
    variable is unset or does not name one (the builds that read it are then
    skipped; their outputs under oracle/_ref/ run without it)."""
    r = os.environ.get("EVX_REFERENCE_ROOT")
    if r and os.path.isdir(os.path.join(r, "plugins")) and os.path.isdir(os.path.join(r, "system", "tmine")):
        return r
    return None


def build() -> None:
    """Compile the oracle (and, where EVX_REFERENCE_ROOT names the reference
    tree, the host build of the reference's Baseline body)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref_root = reference_root()
    if ref_root is None:
        return
    if os.path.isdir(os.path.join(ref_root, "plugins")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_root}"], check=True)
    if os.path.isdir(os.path.join(ref_root, "system", "tmine")):
        # the reference's generated search for each constrained bench query
        from oracle import ref_generated
        ref_generated.build_bench_queries()


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_build_csr.argtypes = [ctypes.c_int64, ctypes.c_int, _i32p, _i32p,
                                       _i32p, _i32p, _i32p, _i32p]
        L.oracle_build_csr.restype = ctypes.c_int
        common = [_i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p,
                  ctypes.c_int, _i32p, _i32p, ctypes.c_int,
                  ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
        L.oracle_count.argtypes = common + [ctypes.c_int, ctypes.POINTER(ctypes.c_uint64),
                                            ctypes.POINTER(OracleStats)]
        L.oracle_count.restype = ctypes.c_int
        L.oracle_count_per_root.argtypes = common + [_u64p, _u64p]
        L.oracle_count_per_root.restype = ctypes.c_int
        L.oracle_enumerate.argtypes = common + [ctypes.c_void_p, ctypes.c_int64,
                                                ctypes.POINTER(ctypes.c_uint64)]
        L.oracle_enumerate.restype = ctypes.c_int
        _lib = L
    return _lib


def ref_lib():
    """The host build of the reference's Baseline body, or None."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB_PATH):
        L = ctypes.CDLL(REF_LIB_PATH)
        L.ref_baseline_count.argtypes = [_i32p, ctypes.c_int, _i32p, _i32p, _i32p, _i32p,
                                         _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_ulonglong)]
        L.ref_baseline_count.restype = ctypes.c_int
        if hasattr(L, "ref_baseline_count_strided"):
            L.ref_baseline_count_strided.argtypes = L.ref_baseline_count.argtypes[:12] + [ctypes.c_int] + \
                L.ref_baseline_count.argtypes[12:]
            L.ref_baseline_count_strided.restype = ctypes.c_int
        _ref = L
    return _ref


# ------------------------------------------------------------------ motif --

def parse_motif(text: str) -> Tuple[List[int], List[int]]:
    """Motif text -> relabeled (mu, mv).

    Lines ``u v t`` are stable-sorted by t; nodes are numbered 0.. in order of
    first appearance (u before v) over the sorted edges
    (``src/core/cpu/Graph.cc:72-96,198-258``).  Blank lines are skipped."""
    rows = []
    for i, line in enumerate(text.splitlines()):
        parts = line.split()
        if not parts:
            continue
        u, v, t = int(parts[0]), int(parts[1]), int(parts[2])
        rows.append((u, v, t, i))
    rows.sort(key=lambda r: r[2])
    ids = {}
    mu, mv = [], []
    for u, v, _, _ in rows:
        for n in (u, v):
            if n not in ids:
                ids[n] = len(ids)
        mu.append(ids[u])
        mv.append(ids[v])
    return mu, mv


def motif_nodes(mu, mv) -> int:
    return max(max(mu), max(mv)) + 1


# ------------------------------------------------------------------ graph --

class Graph:
    """Sorted edge arrays plus stable CSR (the reference's HostGraphData
    content, minus features)."""

    def __init__(self, u, v, t, num_nodes: Optional[int] = None):
        self.u = np.ascontiguousarray(u, dtype=np.int32)
        self.v = np.ascontiguousarray(v, dtype=np.int32)
        self.t = np.ascontiguousarray(t, dtype=np.int32)
        E = self.u.size
        V = int(num_nodes) if num_nodes is not None else (
            int(max(self.u.max(initial=-1), self.v.max(initial=-1))) + 1)
        self.E, self.V = E, V
        self.out_off = np.zeros(V + 1, np.int32)
        self.in_off = np.zeros(V + 1, np.int32)
        self.out_eid = np.zeros(max(E, 1), np.int32)
        self.in_eid = np.zeros(max(E, 1), np.int32)
        if E:
            rc = lib().oracle_build_csr(E, V, self.u, self.v, self.out_off, self.out_eid,
                                        self.in_off, self.in_eid)
            if rc != 0:
                raise ValueError("node id out of range")

    def _args(self):
        u = self.u if self.E else np.zeros(1, np.int32)
        v = self.v if self.E else np.zeros(1, np.int32)
        t = self.t if self.E else np.zeros(1, np.int32)
        return (u, v, t, self.out_off, self.out_eid, self.in_off, self.in_eid)


def _motif_arrays(mu, mv):
    return (np.ascontiguousarray(mu, dtype=np.int32), np.ascontiguousarray(mv, dtype=np.int32))


def default_roots(g: Graph, k: int) -> Tuple[int, int]:
    """The reference's default job: roots [0, E-k+1) (src/core/cpu/data.cc:452-457)."""
    return 0, max(0, g.E - k + 1)


def count(g: Graph, mu, mv, delta: int, roots: Optional[Tuple[int, int]] = None,
          strict_ts: bool = False, threads: int = 0):
    """Return (count, stats dict)."""
    k = len(mu)
    rb, re_ = roots if roots is not None else default_roots(g, k)
    a_mu, a_mv = _motif_arrays(mu, mv)
    out = ctypes.c_uint64(0)
    st = OracleStats()
    rc = lib().oracle_count(*g._args(), k, a_mu, a_mv, int(delta), int(rb), int(re_),
                            int(strict_ts), int(threads), ctypes.byref(out), ctypes.byref(st))
    if rc != 0:
        raise ValueError("motif violates the search precondition")
    return int(out.value), st.as_dict()


def count_per_root(g: Graph, mu, mv, delta: int, roots=None, strict_ts=False):
    k = len(mu)
    rb, re_ = roots if roots is not None else default_roots(g, k)
    a_mu, a_mv = _motif_arrays(mu, mv)
    n = max(re_ - rb, 1)
    counts = np.zeros(n, np.uint64)
    cands = np.zeros(n, np.uint64)
    rc = lib().oracle_count_per_root(*g._args(), k, a_mu, a_mv, int(delta), int(rb), int(re_),
                                     int(strict_ts), counts, cands)
    if rc != 0:
        raise ValueError("motif violates the search precondition")
    return counts[: re_ - rb], cands[: re_ - rb]


def enumerate_rows(g: Graph, mu, mv, delta: int, cap: int, roots=None, strict_ts=False):
    """Return (rows int32[min(cap,total), k] of sorted-edge ids, total)."""
    k = len(mu)
    rb, re_ = roots if roots is not None else default_roots(g, k)
    a_mu, a_mv = _motif_arrays(mu, mv)
    rows = np.zeros((max(cap, 1), k), np.int32)
    tot = ctypes.c_uint64(0)
    rc = lib().oracle_enumerate(*g._args(), k, a_mu, a_mv, int(delta), int(rb), int(re_),
                                int(strict_ts), rows.ctypes.data, int(cap), ctypes.byref(tot))
    if rc != 0:
        raise ValueError("motif violates the search precondition")
    n = min(cap, int(tot.value))
    return rows[:n].copy(), int(tot.value)


def ref_baseline_count(g: Graph, mu, mv, delta: int, roots=None, threads: int = 1, stride: int = 1):
    """Count with the host build of the reference's own Baseline body over
    roots rb, rb + stride, ... below re_ (roots = (rb, re_), default every
    root).  Raises RuntimeError when that build is absent."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference Baseline host build not present")
    k = len(mu)
    rb, re_ = roots if roots is not None else default_roots(g, k)
    eg = getattr(g, "_eg_aos", None)
    if eg is None:
        eg = g._eg_aos = np.stack([g.u, g.v, g.t], axis=1).astype(np.int32).ravel()
    em = np.stack([np.asarray(mu, np.int32), np.asarray(mv, np.int32),
                   np.arange(1, k + 1, dtype=np.int32)], axis=1).ravel()
    out = ctypes.c_ulonglong(0)
    if stride != 1:
        if not hasattr(L, "ref_baseline_count_strided"):
            raise RuntimeError("reference Baseline host build predates root sampling; rebuild it")
        rc = L.ref_baseline_count_strided(eg, g.E, g.in_eid, g.in_off, g.out_eid, g.out_off, em, k,
                                          motif_nodes(mu, mv), int(delta), int(rb), int(re_), int(stride),
                                          int(threads), ctypes.byref(out))
    else:
        rc = L.ref_baseline_count(eg, g.E, g.in_eid, g.in_off, g.out_eid, g.out_off, em, k,
                                  motif_nodes(mu, mv), int(delta), int(rb), int(re_),
                                  int(threads), ctypes.byref(out))
    if rc != 0:
        raise ValueError("motif too large for the Baseline body (<=5 nodes, <=6 edges)")
    return int(out.value)


_ref_gpu = None


def ref_gpu_lib():
    """The reference's Baseline kernel built for sm_100a, or None."""
    global _ref_gpu
    if _ref_gpu is None and os.path.exists(REF_GPU_LIB_PATH):
        L = ctypes.CDLL(REF_GPU_LIB_PATH)
        L.ref_gpu_count.argtypes = [_i32p, ctypes.c_int, _i32p, _i32p, _i32p, _i32p, ctypes.c_int,
                                    _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong),
                                    ctypes.POINTER(ctypes.c_float)]
        L.ref_gpu_count.restype = ctypes.c_int
        _ref_gpu = L
    return _ref_gpu


def ref_gpu_count(g: Graph, mu, mv, delta: int, reps: int = 2):
    """(count, fastest ms of reps launches) of the reference's own Baseline
    kernel on the GPU over every root (work = E - k + 1, as MineJob sets
    it).  Raises RuntimeError when that build is absent."""
    L = ref_gpu_lib()
    if L is None:
        raise RuntimeError("reference Baseline GPU build not present")
    k = len(mu)
    eg = np.stack([g.u, g.v, g.t], axis=1).astype(np.int32).ravel()
    em = np.stack([np.asarray(mu, np.int32), np.asarray(mv, np.int32),
                   np.arange(1, k + 1, dtype=np.int32)], axis=1).ravel()
    out = ctypes.c_ulonglong(0)
    ms = ctypes.c_float(0)
    work = max(0, g.E - k + 1)
    rc = L.ref_gpu_count(eg, g.E, g.in_eid, g.in_off, g.out_eid, g.out_off, g.V, em, k,
                         motif_nodes(mu, mv), int(delta), work, int(reps), ctypes.byref(out), ctypes.byref(ms))
    if rc == -1:
        raise ValueError("motif too large for the Baseline kernel (<=5 nodes, <=6 edges)")
    if rc != 0:
        raise RuntimeError(f"reference Baseline kernel: CUDA error {rc}")
    return int(out.value), float(ms.value)


# ------------------------------------------------------------ brute force --

def brute_force(u, v, t, mu, mv, delta: int, roots=None, strict_ts=False):
    """All k-tuples e0<e1<..<e_{k-1} of edge ids with u(e0)!=v(e0),
    t(ej) <= t(e0)+delta and an injective node map.  Returns the sorted list
    of tuples.  For graphs of a few dozen edges only."""
    E = len(u)
    k = len(mu)
    rb, re_ = roots if roots is not None else (0, max(0, E - k + 1))
    out = []
    for combo in itertools.combinations(range(E), k):
        e0 = combo[0]
        if e0 < rb or e0 >= re_ or u[e0] == v[e0]:
            continue
        tl = int(t[e0]) + delta
        if any(int(t[e]) > tl for e in combo):
            continue
        if strict_ts and any(int(t[combo[i]]) >= int(t[combo[i + 1]]) for i in range(k - 1)):
            continue
        phi = {}
        ok = True
        for j, e in enumerate(combo):
            for a, x in ((mu[j], int(u[e])), (mv[j], int(v[e]))):
                if a in phi:
                    if phi[a] != x:
                        ok = False
                        break
                else:
                    phi[a] = x
            if not ok:
                break
        if ok and len(set(phi.values())) == len(phi):
            out.append(combo)
    return out


# ------------------------------------------------------------ constraints --
def _cons_lib():
    L = lib()
    if not getattr(L, "_cons_ready", False):
        args = [_i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, ctypes.c_void_p, ctypes.c_void_p,
                ctypes.c_int, _i32p, _i32p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64]
        L.oracle_count_constrained.argtypes = args + [ctypes.c_int, ctypes.POINTER(ctypes.c_uint64),
                                                      ctypes.c_void_p]
        L.oracle_count_constrained.restype = ctypes.c_int
        L.oracle_enumerate_constrained.argtypes = args + [ctypes.c_void_p, ctypes.c_int64,
                                                          ctypes.POINTER(ctypes.c_uint64)]
        L.oracle_enumerate_constrained.restype = ctypes.c_int
        L.oracle_prog_eval.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_prog_eval.restype = ctypes.c_int64
        L._cons_ready = True
    return L


def _feat_ptr(a):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data


def count_constrained(g: Graph, mu, mv, delta: int, cons, node_feat=None, edge_feat=None,
                      roots=None, threads: int = 0, stats: Optional[dict] = None) -> int:
    """Constrained count; cons is an everest_b200.constraints.EvxConstraints.
    stats, when given, receives roots / r_reads / candidates (the
    algorithmic-bytes counters of the plain oracle)."""
    k = len(mu)
    rb, re_ = roots if roots is not None else default_roots(g, k)
    a_mu, a_mv = _motif_arrays(mu, mv)
    nf, ef = _feat_ptr(node_feat), _feat_ptr(edge_feat)
    out = ctypes.c_uint64(0)
    st = (ctypes.c_uint64 * 3)()
    rc = _cons_lib().oracle_count_constrained(
        *g._args(), nf[1] if nf else None, ef[1] if ef else None, k, a_mu, a_mv, int(delta),
        ctypes.addressof(cons), int(rb), int(re_), int(threads), ctypes.byref(out), ctypes.addressof(st))
    if rc != 0:
        raise ValueError("motif or constraints violate the search precondition")
    if stats is not None:
        stats.update(roots=int(st[0]), r_reads=int(st[1]), candidates=int(st[2]))
    return int(out.value)


def enumerate_constrained(g: Graph, mu, mv, delta: int, cons, cap: int, node_feat=None,
                          edge_feat=None, roots=None):
    """Return (rows int32[min(cap,total), k] of sorted-edge ids, total)."""
    k = len(mu)
    rb, re_ = roots if roots is not None else default_roots(g, k)
    a_mu, a_mv = _motif_arrays(mu, mv)
    nf, ef = _feat_ptr(node_feat), _feat_ptr(edge_feat)
    rows = np.zeros((max(cap, 1), k), np.int32)
    tot = ctypes.c_uint64(0)
    rc = _cons_lib().oracle_enumerate_constrained(
        *g._args(), nf[1] if nf else None, ef[1] if ef else None, k, a_mu, a_mv, int(delta),
        ctypes.addressof(cons), int(rb), int(re_), rows.ctypes.data, int(cap), ctypes.byref(tot))
    if rc != 0:
        raise ValueError("motif or constraints violate the search precondition")
    n = min(cap, int(tot.value))
    return rows[:n].copy(), int(tot.value)


def prog_eval(prog, variables) -> int:
    """The oracle's interpreter of one program (an EvxProgram)."""
    vals = (ctypes.c_int64 * max(1, len(variables)))(*[int(x) for x in variables])
    return int(_cons_lib().oracle_prog_eval(ctypes.addressof(prog), vals))
