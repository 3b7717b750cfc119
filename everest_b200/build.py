"""In-tree build of the native libraries (sm_100a only).

Outputs (next to this file, git-ignored, shipped with the tree):
  libeverest_b200.so   C ABI (include/everest_b200.h): CUDA kernels + host
                       graph preparation.
  corelib*.so          pybind11 module with the reference's ``corelib`` API.
  libEVX.so            ``getWorker`` plugin (the reference's GPUWorker ABI).

Run ``python -m everest_b200.build`` or call ``build()``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-Wall", "-Wno-unused-function"]

CORE_CU = ["evx_search.cu", "evx_graph.cu", "evx_pairs.cu", "evx_capi.cu", "evx_batch.cu", "evx_static.cu",
           "evx_constrained.cu"]
CORE_CC = ["evx_host.cc"]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _cxx() -> str:
    # the image's /usr/bin toolchain (an alternative gcc wrapper on PATH lacks libgomp specs)
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _newer(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _headers():
    hs = [os.path.join(INCLUDE, "everest_b200.h")]
    for f in os.listdir(CSRC):
        if f.endswith((".cuh", ".h", ".hpp")):
            hs.append(os.path.join(CSRC, f))
    return hs


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build(verbose: bool = False, force: bool = False) -> dict:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _headers()
    jobs = []
    objs = []
    for f in CORE_CU:
        src = os.path.join(CSRC, f)
        if not os.path.exists(src):
            continue
        o = os.path.join(OBJ, f + ".o")
        objs.append(o)
        if force or _newer(o, [src] + hdrs):
            jobs.append([_nvcc(), *ARCH, *NVCC_FLAGS, "-I", INCLUDE, "-c", src, "-o", o])
    for f in CORE_CC:
        src = os.path.join(CSRC, f)
        o = os.path.join(OBJ, f + ".o")
        objs.append(o)
        if force or _newer(o, [src] + hdrs):
            jobs.append([_cxx(), *CXX_FLAGS, "-I", INCLUDE, "-c", src, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    lib = os.path.join(PKG, "libeverest_b200.so")
    if force or jobs or _newer(lib, objs):
        _run([_nvcc(), *ARCH, "-shared", "-o", lib, *objs, "-lcudart", "-lpthread"], verbose)
    out = {"libeverest_b200": lib}
    out.update(_build_corelib(verbose, force, lib))
    return out


def _build_corelib(verbose: bool, force: bool, lib: str) -> dict:
    """pybind11 ``corelib`` module and the ``getWorker`` plugin."""
    src_mod = os.path.join(CSRC, "corelib", "corelib_module.cc")
    src_core = os.path.join(CSRC, "corelib", "corelib_core.cc")
    src_plugin = os.path.join(CSRC, "corelib", "plugin_evx.cc")
    if not os.path.exists(src_mod):
        return {}
    try:
        import pybind11
    except ImportError as e:  # pragma: no cover
        raise RuntimeError("pybind11 is required to build corelib") from e
    hdrs = _headers() + [os.path.join(CSRC, "corelib", "corelib.h")]
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    py_inc = sysconfig.get_paths()["include"]
    ext = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    core_so = os.path.join(PKG, "libevx_corelib.so")
    mod_so = os.path.join(PKG, "corelib" + ext)
    plugin_so = os.path.join(PKG, "libEVX.so")
    rpath = "-Wl,-rpath,$ORIGIN"
    common = [_cxx(), "-O2", "-std=c++17", "-fPIC", "-I", INCLUDE, "-I", cuda_inc]
    if force or _newer(core_so, [src_core, lib] + hdrs):
        _run(common + ["-shared", "-o", core_so, src_core, "-L", PKG, "-leverest_b200", rpath], verbose)
    jobs = []
    if force or _newer(plugin_so, [src_plugin, core_so] + hdrs):
        jobs.append(common + ["-shared", "-o", plugin_so, src_plugin, "-L", PKG, "-levx_corelib",
                              "-leverest_b200", rpath])
    if force or _newer(mod_so, [src_mod, core_so] + hdrs):
        jobs.append(common + ["-shared", "-fvisibility=hidden", "-I", pybind11.get_include(),
                              "-I", py_inc, "-o", mod_so, src_mod, "-L", PKG, "-levx_corelib",
                              "-leverest_b200", rpath])
    with cf.ThreadPoolExecutor(max_workers=2) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    return {"corelib": mod_so, "plugin": plugin_so, "corelib_core": core_so}


if __name__ == "__main__":
    res = build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    for k, v in res.items():
        print(f"{k}: {v}")
