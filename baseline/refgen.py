"""The reference's generated search kernel, built for sm_100a.

Everest compiles one CUDA file per query: KernelGen
(system/tmine/KernelGen.py:112-151) renders it from the templates under
system/templates with warpCentric, warpBalancing and tailExpansion on (the
defaults Everest ships, system/tmine/Query.py:7-16), and the plugin's
GPUWorker runs it (system/templates/GPUWorker/*.snp).  This module renders
that file from a scratch copy of the reference's ``system/`` tree, builds it
for sm_100a with the stand-in headers of refgen_shim.h and the driver
refgen_driver.cu, and runs it through its own GPUWorker on device 0.

It serves as the GPU comparator for the search kernel of this repository
(same queries, same B200) and as a full-size parity check.  Two changes are
made to the rendered host code, both described in refgen_shim.h: a larger
tail-expansion offload buffer (the reference's 2092 * 96 contexts can
overflow on a 148-SM part), and a check that refuses an expansion round
whose int prefix sum would wrap.  The kernels are unchanged.

Building needs the reference tree, named by the environment variable
EVX_REFERENCE_ROOT; the built libraries (baseline/_ref/refgen/, git-ignored)
run without it:

    EVX_REFERENCE_ROOT=<reference checkout> python -m baseline.refgen build
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes
import json
import os
import shutil
import subprocess
import sys
import tempfile
import types
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref", "refgen")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# the #include lines KernelGen writes at the top of every file
# (system/templates/top.snp); refgen_shim.h includes the first four itself and
# stands in for the reference's own two headers
_EXPECTED_INCLUDES = ("<stdio.h>", "<cuda.h>", "<thrust/device_ptr.h>", "<thrust/scan.h>",
                      "/include/helpers.cuh\"", "/include/data.h\"")


def reference_root() -> Optional[str]:
    r = os.environ.get("EVX_REFERENCE_ROOT")
    if r and os.path.isdir(os.path.join(r, "system", "tmine")):
        return r
    return None


def query_key(mu: Sequence[int], mv: Sequence[int]) -> str:
    return "m" + "_".join(f"{a}{b}" for a, b in zip(mu, mv))


def library_path(mu, mv) -> str:
    return os.path.join(OUT, query_key(mu, mv) + ".so")


# ------------------------------------------------------------------ build --

class _KernelGen:
    """KernelGen and Query imported from a scratch copy of system/ (its
    tmine/__init__ imports the compiled corelib, so the package is bypassed)."""

    def __init__(self, ref_root: str):
        self.scratch = tempfile.mkdtemp(prefix="evx-refgen-")
        shutil.copytree(os.path.join(ref_root, "system"), os.path.join(self.scratch, "system"))
        pkg = types.ModuleType("tmine")
        pkg.__path__ = [os.path.join(self.scratch, "system", "tmine")]
        self._saved = {m: mod for m, mod in sys.modules.items() if m == "tmine" or m.startswith("tmine.")}
        for m in self._saved:
            del sys.modules[m]
        sys.modules["tmine"] = pkg
        from tmine import KernelGen as KG, Query as Q  # noqa: E402
        self.KG, self.Q = KG, Q

    def render(self, mu, mv) -> str:
        motif = os.path.join(self.scratch, "motif.txt")
        with open(motif, "w") as f:
            for i, (a, b) in enumerate(zip(mu, mv)):
                f.write(f"{a + 1} {b + 1} {i + 1}\n")
        opts = {"gpu": 1, "warpCentric": True, "warpBalancing": True, "tailExpansion": True}
        cons = {"delta": 0}  # delta is a run-time argument of the generated worker
        Q = self.Q
        q = Q.Query.__new__(Q.Query)
        q.queryFile = {"pattern": motif, "graph": "-", "constraints": cons, "options": opts}
        q.name = "query"
        q.cons = Q.Constraints(cons)
        o = Q.Options()
        o.update(Q.Options(opts))
        q.opts = o
        q.cons.genConsTemplates()
        return self.KG.KernelGen(motif, q).generate()

    def close(self) -> None:
        shutil.rmtree(self.scratch, ignore_errors=True)
        for m in [m for m in sys.modules if m == "tmine" or m.startswith("tmine.")]:
            del sys.modules[m]
        sys.modules.update(self._saved)


def patch(src: str) -> str:
    """Strip the #include lines and apply the two host-side changes."""
    lines = src.split("\n")
    incs = [ln for ln in lines if ln.lstrip().startswith("#include")]
    if len(incs) != len(_EXPECTED_INCLUDES) or not all(
            any(ln.rstrip().endswith(e) for ln in incs) for e in _EXPECTED_INCLUDES):
        raise RuntimeError(f"unexpected includes in the generated file: {incs}")
    body = "\n".join(ln for ln in lines if not ln.lstrip().startswith("#include"))
    n = body.count("2092 * 96")
    if n != 4:
        raise RuntimeError(f"expected 4 uses of the offload size 2092 * 96, found {n}")
    body = body.replace("2092 * 96", "REFGEN_OFFLOAD_CONTEXTS")
    anchor = "auto sump = thrust::inclusive_scan(dev_ptr, dev_ptr + offload_cnt, dev_ptr);"
    if body.count(anchor) != 1:
        raise RuntimeError("expansion scan not found in the generated file")
    body = body.replace(anchor, "REFGEN_CHECK_EXPAND(dev_ptr, offload_cnt)\n    " + anchor)
    return body


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def stale(so: str) -> bool:
    """Whether a built library is missing or older than the driver or shim."""
    if not os.path.exists(so):
        return True
    t = os.path.getmtime(so)
    return any(os.path.getmtime(os.path.join(HERE, f)) > t for f in ("refgen_driver.cu", "refgen_shim.h"))


def _compile(body_path: str, so: str) -> str:
    cmd = [_nvcc(), *ARCH, "-O3", "-std=c++17", "-w", "-Xcompiler", "-fPIC", "-shared", "-cudart", "shared",
           "-I", HERE, f'-DREFGEN_BODY="{body_path}"', "-o", so, os.path.join(HERE, "refgen_driver.cu")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {so}:\n{r.stderr[-4000:]}")
    return so


def build(patterns: Sequence[Tuple[Sequence[int], Sequence[int]]], jobs: int = 0, force: bool = False) -> List[str]:
    """Render and compile one library per distinct motif (delta is a run-time
    argument).  Needs EVX_REFERENCE_ROOT."""
    ref = reference_root()
    if ref is None:
        raise RuntimeError("set EVX_REFERENCE_ROOT to a reference checkout to build the generated kernels")
    os.makedirs(OUT, exist_ok=True)
    todo: Dict[str, Tuple[List[int], List[int]]] = {}
    for mu, mv in patterns:
        key = query_key(mu, mv)
        if force or stale(library_path(mu, mv)):
            todo[key] = (list(mu), list(mv))
    if not todo:
        return []
    kg = _KernelGen(ref)
    try:
        srcs = []
        for key, (mu, mv) in todo.items():
            p = os.path.join(OUT, key + ".inc")
            with open(p, "w") as f:
                f.write(patch(kg.render(mu, mv)))
            srcs.append((p, library_path(mu, mv)))
    finally:
        kg.close()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        return list(ex.map(lambda a: _compile(*a), srcs))


# -------------------------------------------------------------------- run --

class RefGenError(RuntimeError):
    pass


_ip = ctypes.POINTER(ctypes.c_int)


def _bind(lib):
    lib.refgen_graph_upload.argtypes = [_ip, ctypes.c_int, _ip, _ip, _ip, _ip, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, ctypes.c_int]
    lib.refgen_graph_upload.restype = ctypes.c_int
    lib.refgen_graph_free.argtypes = [ctypes.c_void_p]
    lib.refgen_graph_free.restype = None
    lib.refgen_count.argtypes = [ctypes.c_void_p, _ip, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong),
                                 ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, ctypes.c_int]
    lib.refgen_count.restype = ctypes.c_int
    return lib


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


_libs: Dict[str, ctypes.CDLL] = {}


def available(mu, mv) -> bool:
    return os.path.exists(library_path(mu, mv))


def _lib(mu, mv) -> ctypes.CDLL:
    p = library_path(mu, mv)
    if p not in _libs:
        if not os.path.exists(p):
            raise RefGenError(f"generated kernel for {query_key(mu, mv)} not built ({p})")
        _libs[p] = _bind(ctypes.CDLL(p))
    return _libs[p]


def _any_lib() -> ctypes.CDLL:
    """Any built library (each carries the graph upload entry points)."""
    if _libs:
        return next(iter(_libs.values()))
    names = sorted(f for f in os.listdir(OUT) if f.endswith(".so")) if os.path.isdir(OUT) else []
    if not names:
        raise RefGenError(f"no generated kernel built under {OUT}")
    p = os.path.join(OUT, names[0])
    _libs[p] = _bind(ctypes.CDLL(p))
    return _libs[p]


class RefGraph:
    """The reference's HostGraphData arrays on device 0: Eg (AoS u, v, t),
    in/out edge-id lists grouped by node in ascending edge id, and their
    offsets (src/core/gpu/data.cu:124-348)."""

    def __init__(self, u, v, t, in_v, in_r, out_v, out_r, num_vertices: int):
        self._lib = _any_lib()
        eg = np.ascontiguousarray(np.stack([np.asarray(u, np.int32), np.asarray(v, np.int32),
                                            np.asarray(t, np.int32)], axis=1).ravel())
        E = int(np.asarray(u).size)
        arrs = [eg] + [np.ascontiguousarray(a, np.int32) if np.asarray(a).size else np.zeros(1, np.int32)
                       for a in (in_v, in_r, out_v, out_r)]
        if eg.size == 0:
            arrs[0] = np.zeros(3, np.int32)
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = self._lib.refgen_graph_upload(_iptr(arrs[0]), E, _iptr(arrs[1]), _iptr(arrs[2]), _iptr(arrs[3]),
                                           _iptr(arrs[4]), int(num_vertices), ctypes.byref(h), err, 512)
        if rc:
            raise RefGenError(f"graph upload failed ({rc}): {err.value.decode()}")
        self.handle = h
        self.num_edges = E

    @classmethod
    def from_host_graph(cls, h) -> "RefGraph":
        """From the reference's HostGraphData arrays as this library builds
        them (everest_b200.capi.HostGraph: relabeled vertices, Eg AoS)."""
        eg = np.asarray(h.eg, np.int32).reshape(-1, 3)
        return cls(eg[:, 0], eg[:, 1], eg[:, 2], h.in_v, h.in_r, h.out_v, h.out_r, h.num_vertices)

    @classmethod
    def from_oracle_graph(cls, g) -> "RefGraph":
        """From an oracle.Graph (sorted edges plus stable CSR by edge id)."""
        return cls(g.u, g.v, g.t, g.in_eid[:g.E], g.in_off, g.out_eid[:g.E], g.out_off, g.V)

    def free(self) -> None:
        if self.handle:
            self._lib.refgen_graph_free(self.handle)
            self.handle = None


def count(graph: RefGraph, mu, mv, delta: int, beg: int = 0, end: int = -1, reps: int = 1) -> Tuple[int, List[float]]:
    """(count, host ms of each run()) of the reference's generated search."""
    lib = _lib(mu, mv)
    mu_a = np.ascontiguousarray(mu, np.int32)
    mv_a = np.ascontiguousarray(mv, np.int32)
    out = ctypes.c_ulonglong(0)
    ms = (ctypes.c_double * reps)()
    err = ctypes.create_string_buffer(512)
    rc = lib.refgen_count(graph.handle, _iptr(mu_a), _iptr(mv_a), len(mu), int(delta), int(beg), int(end),
                          int(reps), ctypes.byref(out), ms, err, 512)
    if rc:
        raise RefGenError(f"generated search failed ({rc}): {err.value.decode()}")
    return int(out.value), list(ms)


# ----------------------------------------------------------- query sets --

def query_sets() -> Dict[str, List[dict]]:
    """The queries the tests and the bench run on the generated kernels."""
    sys.path.insert(0, ROOT)
    from everest_b200 import workloads
    c3 = workloads.batch_queries()
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        golden = {(tuple(c["mu"]), tuple(c["mv"])) for c in json.load(f)["cases"]}
    sets = {"golden": [{"name": R_key, "mu": list(mu), "mv": list(mv), "delta": 0}
                       for mu, mv in sorted(golden) for R_key in [query_key(mu, mv)]],
            "bursty-7.8m-3edge": workloads.queries("bursty-7.8m-3edge"),
            "c3": [dict(q, name=f"c3-{i:02d}") for i, q in enumerate(c3)],
            "c4-cycle": [{"name": "4-cycle", "mu": [0, 1, 2, 3], "mv": [1, 2, 3, 0], "delta": 86400}],
            "serve-slice": workloads.refgen_serve_slice()}
    return sets


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if not argv or argv[0] != "build":
        print(__doc__)
        return 2
    pats = []
    for qs in query_sets().values():
        for q in qs:
            pats.append((q["mu"], q["mv"]))
    built = build(pats, force="-f" in argv)
    print(f"built {len(built)} generated kernels into {OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
