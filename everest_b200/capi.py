"""ctypes binding of the C ABI (``include/everest_b200.h``).

The native library is required: importing this module on a machine where
``libeverest_b200.so`` has not been built raises immediately (there is no CPU
fallback anywhere in the product path).
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence, Tuple

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("EVX_LIB_PATH") or os.path.join(PKG, "libeverest_b200.so")

EVX_OK = 0
EVX_ERR = {
    -1: "EVX_ERR_INVALID", -2: "EVX_ERR_CUDA", -3: "EVX_ERR_NOMEM", -4: "EVX_ERR_OVERFLOW",
    -5: "EVX_ERR_IO", -6: "EVX_ERR_STATE", -7: "EVX_ERR_TIMEOUT", -8: "EVX_ERR_NODEVICE",
    -9: "EVX_ERR_LIMIT",
}
EVX_ERR_LIMIT = -9
LIMITED = 2**64 - 1  # Batch.result() count of a query stopped at the work limit
FLAG_STRICT_TS = 1
FLAG_EXACT_TOTAL = 2
FLAG_NO_STEAL = 4
FLAG_NO_PAIR_INDEX = 8
FLAG_PAIR_DIR = 16
FLAG_CLOSING_SCAN = 32
FLAG_NO_CLOSING_PRUNE = 64
FLAG_NEW_SCAN = 128
FLAG_LIST_SCAN = 256
FLAG_PER_LANE = 512
FLAG_WARP_SYNC = 1024
FLAG_NO_ROOT_BOUND = 2048
MAX_MOTIF_EDGES = 8

# every symbol include/everest_b200.h declares
EXPORTS = [
    "evx_last_error", "evx_device_count", "evx_edgelist_parse", "evx_graph_build_host",
    "evx_motif_parse", "evx_motif_parse_text", "evx_free", "evx_graph_upload",
    "evx_graph_from_device", "evx_graph_free", "evx_graph_info", "evx_worker_create",
    "evx_worker_destroy", "evx_worker_stream", "evx_worker_take", "evx_worker_run",
    "evx_worker_launch", "evx_worker_result", "evx_worker_enum_rows", "evx_worker_set_tuning",
    "evx_worker_last_stats", "evx_host_register", "evx_host_unregister", "evx_count_static",
    "evx_batch_create", "evx_batch_destroy", "evx_batch_add", "evx_batch_clear", "evx_batch_launch",
    "evx_batch_result", "evx_batch_run", "evx_batch_set_tuning", "evx_batch_last_stats",
    "evx_device_mem_info", "evx_worker_query", "evx_batch_query", "evx_worker_set_limit",
    "evx_batch_set_limit", "evx_graph_set_features", "evx_worker_take_constrained",
]
STATIC_MAX_QUERIES = 256


class EvxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{EVX_ERR.get(code, code)}: {msg}")
        self.code = code


class LimitExceeded(EvxError):
    """A query passed its work limit; ``count`` is the lower bound counted
    before the search stopped."""

    def __init__(self, count: int, limit: int):
        super().__init__(EVX_ERR_LIMIT, f"work limit {limit} exceeded (counted {count} before stopping)")
        self.count = count
        self.limit = limit


_lib = None
_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_PI = ctypes.POINTER(ctypes.c_int)
_PPI = ctypes.POINTER(ctypes.POINTER(ctypes.c_int))
_PI64 = ctypes.POINTER(ctypes.c_int64)
_PU64 = ctypes.POINTER(ctypes.c_uint64)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `python -m everest_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "evx_last_error": ([], ctypes.c_char_p),
            "evx_device_count": ([_PI], _I),
            "evx_device_mem_info": ([_I, _PI64, _PI64], _I),
            "evx_worker_query": ([_P, _PI], _I),
            "evx_batch_query": ([_P, _PI], _I),
            "evx_edgelist_parse": ([ctypes.c_char_p, _PI64, _PPI, _PPI, _PPI, _PPI], _I),
            "evx_graph_build_host": ([_P, _P, _P, _P, _I64, _I64, _PI64, _PI64,
                                      _PPI, _PPI, _PPI, _PPI, _PPI, _PPI], _I),
            "evx_motif_parse": ([ctypes.c_char_p, _PI, _PI, _PI, _PI], _I),
            "evx_motif_parse_text": ([ctypes.c_char_p, _PI, _PI, _PI, _PI], _I),
            "evx_free": ([_P], None),
            "evx_host_register": ([_P, _I64], _I),
            "evx_host_unregister": ([_P], _I),
            "evx_count_static": ([_P, _I, _PI, _PI, _PI, _PI, _I64, _I64, ctypes.c_uint, _P,
                                  _PU64], _I),
            "evx_graph_upload": ([_I, _I64, _I64, _P, _P, _P, _P, _P, _P, _P,
                                  ctypes.POINTER(_P)], _I),
            "evx_graph_from_device": ([_I, _I64, _I64, _P, _P, _P, _P, _P, _P, _P,
                                       ctypes.POINTER(_P)], _I),
            "evx_graph_free": ([_P], _I),
            "evx_graph_info": ([_P, _PI64, _PI64, _PI, _PI64], _I),
            "evx_worker_create": ([_I, _P, ctypes.POINTER(_P)], _I),
            "evx_worker_destroy": ([_P], _I),
            "evx_worker_stream": ([_P, ctypes.POINTER(_P)], _I),
            "evx_worker_take": ([_P, _P, _I, _PI, _PI, _I, _I64, _I64, _I64, ctypes.c_uint], _I),
            "evx_worker_take_constrained": ([_P, _P, _I, _PI, _PI, _I, _I64, _I64, _I64, ctypes.c_uint,
                                             _P], _I),
            "evx_graph_set_features": ([_P, _P, _P], _I),
            "evx_worker_run": ([_P, _PU64], _I),
            "evx_worker_launch": ([_P], _I),
            "evx_worker_result": ([_P, _PU64], _I),
            "evx_worker_enum_rows": ([_P, _I64, _P, _PI64], _I),
            "evx_worker_set_tuning": ([_P, _I, _I, _I, _I, _I], _I),
            "evx_worker_set_limit": ([_P, ctypes.c_uint64], _I),
            "evx_batch_set_limit": ([_P, ctypes.c_uint64], _I),
            "evx_worker_last_stats": ([_P, _PI, ctypes.POINTER(ctypes.c_float)], _I),
            "evx_batch_create": ([_I, _I, _P, ctypes.POINTER(_P)], _I),
            "evx_batch_destroy": ([_P], _I),
            "evx_batch_add": ([_P, _P, _I, _PI, _PI, _I, _I64, _I64, ctypes.c_uint, _PI], _I),
            "evx_batch_clear": ([_P], _I),
            "evx_batch_launch": ([_P], _I),
            "evx_batch_result": ([_P, _PU64, _I], _I),
            "evx_batch_run": ([_P, _PU64, _I], _I),
            "evx_batch_set_tuning": ([_P, _I, _I, _I, _I, _I, _I], _I),
            "evx_batch_last_stats": ([_P, _PI, ctypes.POINTER(ctypes.c_float)], _I),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != EVX_OK:
        msg = lib().evx_last_error()
        raise EvxError(rc, msg.decode() if msg else "")


def device_count() -> int:
    n = ctypes.c_int(0)
    check(lib().evx_device_count(ctypes.byref(n)))
    return n.value


def device_mem_info(device: int = 0):
    """(free, total) device memory in bytes."""
    fr, tot = ctypes.c_int64(0), ctypes.c_int64(0)
    check(lib().evx_device_mem_info(int(device), ctypes.byref(fr), ctypes.byref(tot)))
    return fr.value, tot.value


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _take_int_array(p, n: int) -> np.ndarray:
    arr = np.ctypeslib.as_array(p, shape=(max(n, 1),))[:n].copy()
    lib().evx_free(ctypes.cast(p, ctypes.c_void_p))
    return arr


# ----------------------------------------------------------- host data --

def edgelist_parse(path: str):
    """Parse a ``u v t`` file; return (u, v, t, ids) int32 arrays sorted by t
    (stable) with ids = original line index."""
    n = ctypes.c_int64(0)
    pu, pv, pt, pi = (ctypes.POINTER(ctypes.c_int)() for _ in range(4))
    check(lib().evx_edgelist_parse(path.encode(), ctypes.byref(n), ctypes.byref(pu),
                                   ctypes.byref(pv), ctypes.byref(pt), ctypes.byref(pi)))
    E = n.value
    return (_take_int_array(pu, E), _take_int_array(pv, E), _take_int_array(pt, E),
            _take_int_array(pi, E))


def host_register(arr: np.ndarray) -> None:
    """Page-lock a numpy array (uploads from it become async DMA)."""
    check(lib().evx_host_register(_ptr(arr), arr.nbytes))


def host_unregister(arr: np.ndarray) -> None:
    check(lib().evx_host_unregister(_ptr(arr)))


class HostGraph:
    """Host-format graph arrays (the reference's HostGraphData content)."""

    def __init__(self, num_edges, num_vertices, eg, out_v, in_v, out_r, in_r, euid, name=""):
        self.num_edges = int(num_edges)
        self.num_vertices = int(num_vertices)
        self.eg, self.out_v, self.in_v = eg, out_v, in_v
        self.out_r, self.in_r, self.euid = out_r, in_r, euid
        self.name = name

    def original_vertex_ids(self, u, v, beg: int = 0) -> np.ndarray:
        """Input vertex id of every relabeled vertex, given the input edge
        arrays this graph was built from, starting at edge beg (node
        features follow this map)."""
        eg = self.eg.reshape(-1, 3)
        src = np.asarray(u)[beg:beg + self.num_edges]
        dst = np.asarray(v)[beg:beg + self.num_edges]
        orig = np.full(self.num_vertices, -1, np.int64)
        orig[eg[:, 0]] = src
        orig[eg[:, 1]] = dst
        return orig

    @property
    def total_bytes(self) -> int:
        return 24 * self.num_edges + 8 * (self.num_vertices + 1)

    def arrays(self):
        return [self.eg, self.out_v, self.in_v, self.out_r, self.in_r, self.euid]

    def pin(self) -> "HostGraph":
        """Page-lock every array (idempotent)."""
        if not getattr(self, "_pinned", False):
            for a in self.arrays():
                if a.nbytes:
                    host_register(a)
            self._pinned = True
        return self

    def unpin(self) -> None:
        if getattr(self, "_pinned", False):
            for a in self.arrays():
                if a.nbytes:
                    host_unregister(a)
            self._pinned = False


def graph_build_host(u, v, t, ids=None, beg: int = 0, end: Optional[int] = None,
                     name: str = "") -> HostGraph:
    u = np.ascontiguousarray(u, np.int32)
    v = np.ascontiguousarray(v, np.int32)
    t = np.ascontiguousarray(t, np.int32)
    ids = None if ids is None else np.ascontiguousarray(ids, np.int32)
    if end is None:
        end = u.size
    E, V = ctypes.c_int64(0), ctypes.c_int64(0)
    outs = [ctypes.POINTER(ctypes.c_int)() for _ in range(6)]
    check(lib().evx_graph_build_host(_ptr(u), _ptr(v), _ptr(t), _ptr(ids), int(beg), int(end),
                                     ctypes.byref(E), ctypes.byref(V),
                                     *[ctypes.byref(o) for o in outs]))
    e, n = E.value, V.value
    eg = _take_int_array(outs[0], 3 * e)
    ov = _take_int_array(outs[1], e)
    iv = _take_int_array(outs[2], e)
    orr = _take_int_array(outs[3], n + 1)
    irr = _take_int_array(outs[4], n + 1)
    eu = _take_int_array(outs[5], e)
    return HostGraph(e, n, eg, ov, iv, orr, irr, eu, name)


def motif_parse_text(text: str) -> Tuple[list, list, int]:
    k = ctypes.c_int(0)
    nn = ctypes.c_int(0)
    mu = (ctypes.c_int * MAX_MOTIF_EDGES)()
    mv = (ctypes.c_int * MAX_MOTIF_EDGES)()
    check(lib().evx_motif_parse_text(text.encode(), ctypes.byref(k), mu, mv, ctypes.byref(nn)))
    return list(mu[: k.value]), list(mv[: k.value]), nn.value


def motif_parse(path: str) -> Tuple[list, list, int]:
    k = ctypes.c_int(0)
    nn = ctypes.c_int(0)
    mu = (ctypes.c_int * MAX_MOTIF_EDGES)()
    mv = (ctypes.c_int * MAX_MOTIF_EDGES)()
    check(lib().evx_motif_parse(path.encode(), ctypes.byref(k), mu, mv, ctypes.byref(nn)))
    return list(mu[: k.value]), list(mv[: k.value]), nn.value


# --------------------------------------------------------- device graph --

class DeviceGraph:
    """A graph resident on one device (owns the device memory)."""

    def __init__(self, host: HostGraph, device: int = 0, stream: Optional[int] = None):
        h = ctypes.c_void_p()
        check(lib().evx_graph_upload(int(device), host.num_edges, host.num_vertices,
                                     _ptr(host.eg), _ptr(host.out_v), _ptr(host.in_v),
                                     _ptr(host.out_r), _ptr(host.in_r), _ptr(host.euid),
                                     ctypes.c_void_p(stream) if stream else None,
                                     ctypes.byref(h)))
        self._h = h
        self.device = device
        self.num_edges = host.num_edges
        self.num_vertices = host.num_vertices
        self.name = host.name

    @classmethod
    def from_device(cls, device, num_edges, num_vertices, eg_d, out_v_d, in_v_d, out_r_d,
                    in_r_d, euid_d, stream=None):
        self = cls.__new__(cls)
        h = ctypes.c_void_p()
        check(lib().evx_graph_from_device(int(device), int(num_edges), int(num_vertices),
                                          ctypes.c_void_p(eg_d), ctypes.c_void_p(out_v_d),
                                          ctypes.c_void_p(in_v_d), ctypes.c_void_p(out_r_d),
                                          ctypes.c_void_p(in_r_d),
                                          ctypes.c_void_p(euid_d) if euid_d else None,
                                          ctypes.c_void_p(stream) if stream else None,
                                          ctypes.byref(h)))
        self._h = h
        self.device = device
        self.num_edges = int(num_edges)
        self.num_vertices = int(num_vertices)
        self.name = ""
        return self

    @property
    def handle(self):
        return self._h

    def set_features(self, node_features=None, edge_features=None) -> None:
        """Node features (int32 per vertex id) and edge features (int32 per
        sorted edge id) for constraint predicates and filters."""
        nf = None if node_features is None else np.ascontiguousarray(node_features, dtype=np.int32)
        ef = None if edge_features is None else np.ascontiguousarray(edge_features, dtype=np.int32)
        if nf is not None and nf.size != self.num_vertices:
            raise ValueError(f"{nf.size} node features for {self.num_vertices} vertices")
        if ef is not None and ef.size != self.num_edges:
            raise ValueError(f"{ef.size} edge features for {self.num_edges} edges")
        check(lib().evx_graph_set_features(self._h, _ptr(nf), _ptr(ef)))

    def info(self):
        E, V, B = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        d = ctypes.c_int()
        check(lib().evx_graph_info(self._h, ctypes.byref(E), ctypes.byref(V), ctypes.byref(d),
                                   ctypes.byref(B)))
        return {"num_edges": E.value, "num_vertices": V.value, "device": d.value,
                "device_bytes": B.value}

    def free(self):
        if getattr(self, "_h", None):
            lib().evx_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def count_static(graph: "DeviceGraph", queries, beg: int = 0, end: int = -1, flags: int = 0,
                 stream: Optional[int] = None):
    """Count queries [(mu, mv, delta), ...] through the allocation-free entry
    point (for callers that cannot allocate device memory at query time)."""
    nq = len(queries)
    ks = [len(q[0]) for q in queries]
    mu = [x for q in queries for x in q[0]]
    mv = [x for q in queries for x in q[1]]
    a_k = (ctypes.c_int * max(nq, 1))(*ks)
    a_mu = (ctypes.c_int * max(len(mu), 1))(*mu)
    a_mv = (ctypes.c_int * max(len(mv), 1))(*mv)
    a_d = (ctypes.c_int * max(nq, 1))(*[int(q[2]) for q in queries])
    out = (ctypes.c_uint64 * max(nq, 1))()
    check(lib().evx_count_static(graph.handle, nq, a_k, a_mu, a_mv, a_d, int(beg), int(end),
                                 int(flags), ctypes.c_void_p(stream) if stream else None, out))
    return [int(out[i]) for i in range(nq)]


# --------------------------------------------------------------- worker --

class Worker:
    """Per-device search worker (the reference's GPUWorker)."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        h = ctypes.c_void_p()
        check(lib().evx_worker_create(int(device), ctypes.c_void_p(stream) if stream else None,
                                      ctypes.byref(h)))
        self._h = h
        self.device = device
        self.k = 0
        self.enum_cap = 0

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        check(lib().evx_worker_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def set_tuning(self, block=256, blocks_per_sm=0, roots_per_fetch=32, steal_interval=16,
                   min_split=2):
        check(lib().evx_worker_set_tuning(self._h, block, blocks_per_sm, roots_per_fetch,
                                          steal_interval, min_split))

    def take(self, graph: DeviceGraph, mu: Sequence[int], mv: Sequence[int], delta: int,
             beg: int = 0, end: int = -1, enum_cap: int = 0, flags: int = 0, constraints=None):
        """Bind a job; constraints (an everest_b200.constraints.Constraints or
        its EvxConstraints struct) selects the constrained search."""
        k = len(mu)
        a_mu = (ctypes.c_int * k)(*mu)
        a_mv = (ctypes.c_int * k)(*mv)
        if constraints is None:
            check(lib().evx_worker_take(self._h, graph.handle, k, a_mu, a_mv, int(delta), int(beg),
                                        int(end), int(enum_cap), int(flags)))
        else:
            st = constraints.to_struct() if hasattr(constraints, "to_struct") else constraints
            check(lib().evx_worker_take_constrained(self._h, graph.handle, k, a_mu, a_mv, int(delta),
                                                    int(beg), int(end), int(enum_cap), int(flags),
                                                    ctypes.byref(st)))
        self.k = k
        self.enum_cap = int(enum_cap)

    def set_limit(self, max_work: int) -> None:
        """Work limit of later jobs (0 = none), in adjacency records examined
        inside their time windows; run()/result() raise LimitExceeded for a
        query whose work passes it (an enumeration keeps its rows so far)."""
        check(lib().evx_worker_set_limit(self._h, int(max_work)))
        self.limit = int(max_work)

    def _count(self, rc: int, c: ctypes.c_uint64) -> int:
        if rc == EVX_ERR_LIMIT:
            raise LimitExceeded(int(c.value), getattr(self, "limit", 0))
        check(rc)
        return int(c.value)

    def run(self) -> int:
        c = ctypes.c_uint64(0)
        return self._count(lib().evx_worker_run(self._h, ctypes.byref(c)), c)

    def launch(self) -> None:
        check(lib().evx_worker_launch(self._h))

    def result(self) -> int:
        c = ctypes.c_uint64(0)
        return self._count(lib().evx_worker_result(self._h, ctypes.byref(c)), c)

    def done(self) -> bool:
        """True once the launched search has finished (never blocks)."""
        d = ctypes.c_int(0)
        check(lib().evx_worker_query(self._h, ctypes.byref(d)))
        return bool(d.value)

    def enum_rows(self, n: int) -> np.ndarray:
        n = max(0, int(n))
        buf = np.zeros((max(n, 1), max(self.k, 1)), np.int32)
        wr = ctypes.c_int64(0)
        check(lib().evx_worker_enum_rows(self._h, n, _ptr(buf), ctypes.byref(wr)))
        return buf[: wr.value].copy()

    def last_stats(self):
        n = ctypes.c_int()
        ms = ctypes.c_float()
        check(lib().evx_worker_last_stats(self._h, ctypes.byref(n), ctypes.byref(ms)))
        return {"kernel_launches": n.value, "device_ms": ms.value}

    def close(self):
        if getattr(self, "_h", None):
            lib().evx_worker_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# -------------------------------------------------------------- batches --

class Batch:
    """Many count queries on one resident graph in one persistent launch."""

    def __init__(self, device: int = 0, max_queries: int = 1024, stream: Optional[int] = None):
        h = ctypes.c_void_p()
        check(lib().evx_batch_create(int(device), int(max_queries),
                                     ctypes.c_void_p(stream) if stream else None, ctypes.byref(h)))
        self._h = h
        self.n = 0

    def set_tuning(self, tile_roots=256, blocks_per_sm=0, steal_interval=16, min_split=2, use_graph=True):
        check(lib().evx_batch_set_tuning(self._h, tile_roots, blocks_per_sm, steal_interval, min_split,
                                         1 if use_graph else 0, 0))

    def set_limit(self, max_work: int) -> None:
        """Work limit per query (0 = none); result() then holds LIMITED for
        each query that was stopped."""
        check(lib().evx_batch_set_limit(self._h, int(max_work)))
        self.limit = int(max_work)

    def add(self, graph: DeviceGraph, mu, mv, delta, beg=0, end=-1, flags=0) -> int:
        k = len(mu)
        idx = ctypes.c_int(0)
        check(lib().evx_batch_add(self._h, graph.handle, k, (ctypes.c_int * k)(*mu), (ctypes.c_int * k)(*mv),
                                  int(delta), int(beg), int(end), int(flags), ctypes.byref(idx)))
        self.n += 1
        return idx.value

    def clear(self):
        check(lib().evx_batch_clear(self._h))
        self.n = 0

    def launch(self):
        check(lib().evx_batch_launch(self._h))

    def result(self):
        out = (ctypes.c_uint64 * max(self.n, 1))()
        check(lib().evx_batch_result(self._h, out, self.n))
        return [int(out[i]) for i in range(self.n)]

    def run(self):
        self.launch()
        return self.result()

    def done(self) -> bool:
        d = ctypes.c_int(0)
        check(lib().evx_batch_query(self._h, ctypes.byref(d)))
        return bool(d.value)

    def last_stats(self):
        n = ctypes.c_int()
        ms = ctypes.c_float()
        check(lib().evx_batch_last_stats(self._h, ctypes.byref(n), ctypes.byref(ms)))
        return {"kernel_launches": n.value, "device_ms": ms.value}

    def close(self):
        if getattr(self, "_h", None):
            lib().evx_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
