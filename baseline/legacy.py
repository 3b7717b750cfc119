"""The reference's legacy ablation plugins, built for sm_100a.

Everest ships, beside its generated kernel, hand-written plugins that add one
optimisation at a time (plugins/GPUWorker{U0,U1,U1B,U2,U3,U3B}.cu; run by
system/legacy.py, the "Figure 10" ablation of README.md:284-304).  This
module compiles each plugin file as it lies in the reference tree
(EVX_REFERENCE_ROOT) for sm_100a, with the stand-in corelib headers of
refgen_shim.h and the driver refgen_driver.cu, into baseline/_ref/legacy/
(git-ignored), and runs it through its own GPUWorker on device 0 -- the same
path as baseline/refgen.py.

Changes to the plugin text, host side only: its #include lines are replaced
by the shim; U3 and U3B, which carry the tail-expansion offload buffer of
2092 * 96 contexts, get the larger buffer and the int-overflow check before
the expansion scan that refgen_shim.h describes.  The plugins keep every
motif's state in fixed arrays of 5 nodes and 5 edges (MapMg[5],
Estackbeg[4], m0..m4), so run() refuses larger motifs.

    EVX_REFERENCE_ROOT=<reference checkout> python -m baseline.legacy build
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes
import os
import subprocess
import sys
from typing import Dict, List, Tuple

import numpy as np

from . import refgen as R

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref", "legacy")
PLUGINS = ("U0", "U1", "U1B", "U2", "U3", "U3B")
MAX_NODES = 5
MAX_EDGES = 5


def library_path(name: str) -> str:
    return os.path.join(OUT, f"lib{name}.so")


def available(name: str) -> bool:
    return os.path.exists(library_path(name))


def patch(name: str, src: str) -> str:
    lines = src.split("\n")
    body = "\n".join(ln for ln in lines if not ln.lstrip().startswith("#include"))
    if name in ("U3", "U3B"):
        n = body.count("2092 * 96")
        if n != 4:
            raise RuntimeError(f"{name}: expected 4 uses of the offload size 2092 * 96, found {n}")
        body = body.replace("2092 * 96", "REFGEN_OFFLOAD_CONTEXTS")
        anchor = "auto sump = thrust::inclusive_scan(dev_ptr, dev_ptr + offload_cnt, dev_ptr);"
        if body.count(anchor) != 1:
            raise RuntimeError(f"{name}: expansion scan not found")
        body = body.replace(anchor, "REFGEN_CHECK_EXPAND(dev_ptr, offload_cnt)\n      " + anchor)
    elif "2092" in body:
        raise RuntimeError(f"{name}: unexpected offload buffer")
    return body


def build(force: bool = False) -> List[str]:
    ref = R.reference_root()
    if ref is None:
        raise RuntimeError("set EVX_REFERENCE_ROOT to a reference checkout to build the legacy plugins")
    os.makedirs(OUT, exist_ok=True)
    jobs = []
    for name in PLUGINS:
        so = library_path(name)
        if not force and not R.stale(so):
            continue
        with open(os.path.join(ref, "plugins", f"GPUWorker{name}.cu")) as f:
            body = patch(name, f.read())
        inc = os.path.join(OUT, f"{name}.inc")
        with open(inc, "w") as f:
            f.write(body)
        jobs.append((inc, so))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        return list(ex.map(lambda a: R._compile(*a), jobs))


_libs: Dict[str, ctypes.CDLL] = {}


def _lib(name: str) -> ctypes.CDLL:
    p = library_path(name)
    if p not in _libs:
        if not os.path.exists(p):
            raise R.RefGenError(f"legacy plugin {name} not built ({p})")
        _libs[p] = R._bind(ctypes.CDLL(p))
    return _libs[p]


def count(name: str, graph: R.RefGraph, mu, mv, delta: int, beg: int = 0, end: int = -1,
          reps: int = 1) -> Tuple[int, List[float]]:
    """(count, host ms of each run()) of the legacy plugin `name`."""
    if len(mu) > MAX_EDGES or max(max(mu), max(mv)) + 1 > MAX_NODES:
        raise ValueError(f"the legacy plugins hold at most {MAX_NODES} nodes and {MAX_EDGES} edges")
    lib = _lib(name)
    mu_a = np.ascontiguousarray(mu, np.int32)
    mv_a = np.ascontiguousarray(mv, np.int32)
    out = ctypes.c_ulonglong(0)
    ms = (ctypes.c_double * reps)()
    err = ctypes.create_string_buffer(512)
    rc = lib.refgen_count(graph.handle, R._iptr(mu_a), R._iptr(mv_a), len(mu), int(delta), int(beg), int(end),
                          int(reps), ctypes.byref(out), ms, err, 512)
    if rc:
        raise R.RefGenError(f"legacy plugin {name} failed ({rc}): {err.value.decode()}")
    return int(out.value), list(ms)


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if not argv or argv[0] != "build":
        print(__doc__)
        return 2
    built = build(force="-f" in argv)
    print(f"built {len(built)} legacy plugins into {OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
