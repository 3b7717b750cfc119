#!/usr/bin/env python
"""Benchmark of the temporal-motif search on B200.

Workload (default ``bursty-7.8m-3edge``): a seeded synthetic temporal graph
with 1.1M nodes and 7.8M edges (power-law out-degree, exponent 2.1; bursty
timestamps over 2.3e8 s), and every connected 3-edge pattern on 2-3 nodes
(36, by rule), each run separately as its own count query with
delta = 86400.  One step = the 36 queries.

Metric: motif matches per second (whole job).  ``value`` is device time with
the graph resident in HBM (CUDA events on the launching stream, L2 flushed
before every step); ``e2e`` goes through the public API from pinned host
arrays: graph upload (host->device + on-device packing), the 36 queries and
the 36 counts read back, every step.

Beside the headline (N = 1, rank 0), the same line carries:
  c1                    the 200k-edge triangle on the GPU and on the host;
  four_cycle            the 4-cycle on the bench graph: kernel time and its
                        effective rate against the measured HBM bandwidth;
  reference_gpu_kernel  the reference's own generated kernel for sm_100a
                        (baseline/refgen.py) on the same 36 queries;
  enumerate             the 36M-edge 4-cycle at cap 1e6 (rows checked);
  batch                 the 64-query mix over the whole 36M-edge graph,
                        batched vs one at a time, every result exact;
  serve                 the serving stream (two resident graphs), served vs
                        one at a time: queries/s, and p50/p99/p99.9 under
                        Poisson arrivals beside a FIFO server's;
  cpu_baseline          the reference's Baseline body on the host cores.

``--impl reference`` times the reference's own CPU implementation of the
path: its legacy Baseline search body (plugins/GPUWorkerBaseline.cu) built
for the host (oracle/_ref), on all host cores, over every 16th root of each
query of the same workload.  When that build is absent, the C restatement
of the same semantics (oracle/) stands in.

Multi-GPU: the path does not shard on one-GPU deployments; N ranks run N
independent replicas (weak scaling), timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "motif matches/s (per-query count kernels, 36 three-edge motifs)"
UNIT = "matches/s"
WORKLOAD = "bursty-7.8m-3edge"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="evx", choices=["evx", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the legs beside the headline step (reference GPU kernel, enumeration, "
                         "batch, serve)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="default launch parameters instead of per-query autotuned ones")
    ap.add_argument("--single-query", type=int, default=-1,
                    help="profiling aid: run only query I of the workload --reps times and exit")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--motif", default="",
                    help="profiling aid: run this motif (edges a-b separated by commas, nodes numbered by first "
                         "appearance, e.g. 0-1,1-2,2-3,3-0) on the workload's graph --reps times and exit")
    ap.add_argument("--delta", type=int, default=86400, help="with --motif: the time window")
    ap.add_argument("--constrained-query", default="",
                    help="profiling aid: run this constrained bench query (M4-no, M4-v, M4-t, M4-all, M4-f) on "
                         "the 7.8M-edge graph with its features --reps times and exit")
    ap.add_argument("--flags", type=int, default=0, help="with --motif / --constrained-query: EVX_FLAG_* bits")
    ap.add_argument("--mode", default="single", choices=["single", "batch", "serve", "enumerate", "constrained"],
                    help="single: the 36-query per-query-kernel step (default); batch: 64 mixed queries "
                         "in one persistent launch per motif size vs the same queries one at a time; serve: "
                         "the serving loop (saturated and Poisson arrivals) vs one at a time; enumerate: "
                         "the 36M-edge 4-cycle at cap 1e6 with a host check of the rows; constrained: the "
                         "reference's node / temporal / anti-edge / filter query shapes on the 7.8M graph")
    ap.add_argument("--queries", type=int, default=0, help="batch/serve: number of queries")
    ap.add_argument("--window", type=int, default=0,
                    help="batch/serve: roots per query (a random time window of the edge list); batch: "
                         "0 = every root of the graph (default)")
    ap.add_argument("--serve-slots", default="64,2,2,2,1.0,2,2",
                    help="serve: max queries per batch, batches in flight, enumeration slots, "
                         "blocks per SM of an enumeration (0 = all), share of a batch kernel's blocks, "
                         "heavy slots, blocks per SM of a heavy query beside other work")
    ap.add_argument("--limit", type=float, default=None,
                    help="work limit per query, in adjacency records examined inside their time windows. "
                         "batch (default 0 = none, every result exact): stopped queries are flagged in both "
                         "arms; serve (default 3e7): queries past it leave the shared batches for heavy slots")
    return ap.parse_args()


def workload_stats(name):
    p = os.path.join(ROOT, "tests", "golden", "workload_stats.json")
    with open(p) as f:
        return json.load(f)[name]


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes (read + write) of the search kernel over one timed step
    (its 36 launches, the unit `roofline.achieved` is computed on) from the
    committed ncu summary (a line 'traffic_bytes_per_step: N'), or None."""
    p = os.path.join(ROOT, "profiles", "search_kernel_bursty-7.8m.md")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.strip().startswith("traffic_bytes_per_step:"):
                try:
                    return float(line.split(":", 1)[1].strip().split()[0])
                except ValueError:
                    return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, p in zip(names, parts[2:6]):
                if p.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local, dist


def max_over_ranks(value: float, dist, device=None) -> float:
    """Max of a per-rank value over all ranks (identity on one rank)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------- CPU reference --

CPU_STRIDE = 16        # the CPU legs time every 16th root of each query
CPU_STRIDE_1T = 256    # the single-thread figure: every 256th root


def host_info() -> dict:
    """Host cores and CPU model of the machine the CPU legs run on."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        usable = os.cpu_count() or 1
    return {"nproc": os.cpu_count() or 1, "usable_cores": usable, "cpu_model": model}


def workload_config(wname) -> dict:
    """The workload the bench line is quoted on (identical in both arms)."""
    from everest_b200 import synth
    stats = workload_stats(wname)
    spec = synth.SPECS[stats["graph"]]
    return {"workload": "bursty-7.8m-3edge: 1.1M nodes, 7.8M edges, 36 three-edge motifs "
                        "run separately, delta 86400, count",
            "graph_edges": spec.num_edges, "graph_vertices": spec.num_nodes,
            "queries_per_step": len(stats["queries"]),
            "matches_per_step": sum(r["count"] for r in stats["queries"]),
            "l2": "GPU arm: flushed before every step (256 MB write); CPU arm: not applicable",
            "parallelism": "replicas (one GPU per query stream; no data-path collective)"}


_cpu_graphs = {}


def cpu_reference(wname, stride, threads):
    """Time the reference's own CPU path (host build of its Baseline body)
    over roots 0, stride, 2 stride, ... of every query of the workload (an
    even sample of the whole time range); returns (matches, seconds, kind,
    roots sampled per query)."""
    from oracle import oracle as O
    from everest_b200 import synth, workloads
    spec = synth.SPECS[workload_stats(wname)["graph"]]
    if spec.name not in _cpu_graphs:
        u, v, t = synth.load_or_generate(spec.name)
        _cpu_graphs[spec.name] = O.Graph(u, v, t, spec.num_nodes)
    g = _cpu_graphs[spec.name]
    kind = "reference" if O.ref_lib() is not None else "port"
    total, n = 0, 0
    t0 = time.perf_counter()
    for q in workloads.queries(wname):
        work = max(0, g.E - len(q["mu"]) + 1)
        n = (work + stride - 1) // stride
        if kind == "reference":
            total += O.ref_baseline_count(g, q["mu"], q["mv"], q["delta"], roots=(0, work),
                                          threads=threads, stride=stride)
        else:
            # the oracle takes contiguous ranges: the same roots one by one
            total += sum(O.count(g, q["mu"], q["mv"], q["delta"], roots=(r, r + 1), threads=1)[0]
                         for r in range(0, work, stride))
    return total, time.perf_counter() - t0, kind, n


def cpu_sample_text(stride, threads, n):
    return (f"every {stride}th root ({n} per query, spread over the whole time range) of each of the 36 "
            f"queries on the 7.8M-edge graph, {threads} threads; rate = sampled matches / time")


def run_reference_arm(args):
    world, rank, local, dist = dist_setup(args.gpus)
    if rank != 0:
        return 0
    threads = host_info()["usable_cores"]
    times, matches = [], 0
    kind, n = "reference", 0
    for i in range(args.warmup + args.steps):
        m, dt, kind, n = cpu_reference(args.workload, CPU_STRIDE, threads)
        if i >= args.warmup:
            times.append(dt)
            matches = m
    sec = sum(times) / len(times)
    val = matches / sec
    sample = cpu_sample_text(CPU_STRIDE, threads, n)
    line = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic (seeded generator; public graphs unavailable offline)",
            "impl": "reference",
            "config": workload_config(args.workload),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": sample, "host": host_info()},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# -------------------------------------------------------------- GPU arm --

def run_gpu_arm(args):
    import torch
    from everest_b200 import capi, synth, workloads

    world, rank, local, dist = dist_setup(args.gpus)
    dev = local
    torch.cuda.set_device(dev)
    stats = workload_stats(args.workload)
    spec = synth.SPECS[stats["graph"]]
    qs = workloads.queries(args.workload)
    want = {r["name"]: r["count"] for r in stats["queries"]}
    bytes_alg = sum(r["bytes_alg"] for r in stats["queries"])
    cands = sum(r["candidates"] for r in stats["queries"])  # edges visited by the serial semantics

    u, v, t = synth.load_or_generate(spec.name)
    host = capi.graph_build_host(u, v, t, name=spec.name)
    host.pin()
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    dg = capi.DeviceGraph(host, dev, sh)
    workers = [capi.Worker(dev, sh) for _ in qs]
    flags = [0] * len(qs)
    tuned = {}
    if not args.no_autotune:
        # per-query launch parameters, tuned on a root sample before timing
        from everest_b200 import autotune
        tuner = autotune.Autotuner(dev, sample_roots=0)  # each candidate timed on the whole query
        for i, (w, q) in enumerate(zip(workers, qs)):
            cfg = tuner.tune(dg, q["mu"], q["mv"], q["delta"], w)
            flags[i] = autotune.Autotuner.apply(w, cfg)
            tuned[q["name"]] = {k: cfg[k] for k in ("blocks_per_sm", "steal_interval", "min_split", "flags")}
    for w, q, f in zip(workers, qs, flags):
        w.take(dg, q["mu"], q["mv"], q["delta"], 0, -1, 0, f)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def device_step():
        with torch.cuda.stream(stream):
            flush.zero_()  # L2 flush (256 MB > 126 MB L2), outside the timed region
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            for w in workers:
                w.launch()
            ev1.record(stream)
        counts = [w.result() for w in workers]
        kms = sum(w.last_stats()["device_ms"] for w in workers)
        launches = sum(w.last_stats()["kernel_launches"] for w in workers)
        return ev0.elapsed_time(ev1), counts, kms, launches

    for _ in range(args.warmup):
        _, counts, _, _ = device_step()
    for q, c in zip(qs, counts):
        if c != want[q["name"]]:
            raise SystemExit(f"count mismatch on {q['name']}: {c} != {want[q['name']]}")
    barrier()
    step_ms, kern_ms, launches = [], [], 0
    with ClockSampler(dev) as clk:
        for _ in range(args.steps):
            # an NVTX range per timed step, so that ncu can capture exactly
            # its launches (--nvtx --nvtx-include timed_step/)
            torch.cuda.nvtx.range_push("timed_step")
            ms, counts, kms, nl = device_step()
            torch.cuda.nvtx.range_pop()
            per_query_ms = {q["name"]: round(w.last_stats()["device_ms"], 3) for q, w in zip(qs, workers)}
            step_ms.append(ms)
            kern_ms.append(kms)
            launches += nl
    barrier()
    total_ms = max_over_ranks(sum(step_ms), dist, f"cuda:{dev}")
    matches = sum(counts)
    ms_per_step = total_ms / args.steps
    value = world * matches / (ms_per_step / 1e3)

    # ---- end to end through the public API from pinned host arrays
    def e2e_step():
        with torch.cuda.stream(stream):
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            g2 = capi.DeviceGraph(host, dev, sh)
            for w, q, f in zip(workers, qs, flags):
                w.take(g2, q["mu"], q["mv"], q["delta"], 0, -1, 0, f)
                w.launch()
            cs = [w.result() for w in workers]
            ev1.record(stream)
        torch.cuda.synchronize(dev)
        ms = ev0.elapsed_time(ev1)
        g2.free()
        return ms, cs

    for _ in range(min(args.warmup, 2)):
        e2e_step()
    barrier()
    e_ms = []
    for _ in range(args.steps):
        ms, cs = e2e_step()
        e_ms.append(ms)
    barrier()
    e_total = max_over_ranks(sum(e_ms), dist, f"cuda:{dev}")
    e2e_val = world * sum(cs) / (e_total / args.steps / 1e3)
    h2d = host.total_bytes + sum(8 * len(q["mu"]) for q in qs)
    d2h = 8 * len(qs)

    peak, peak_kind = measured_peaks()
    kern_avg_ms = sum(kern_ms) / len(kern_ms)
    achieved = bytes_alg / (kern_avg_ms / 1e3) / 1e9
    traffic = profile_traffic()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator with the named shapes; public graphs unavailable offline)",
        "config": workload_config(args.workload),
        "replicas": world,
        "autotune": "per-query, candidates timed on the whole query, outside the timed region"
        if tuned else "off",
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e_total / args.steps},
        "gpu_launches": launches,
        "per_query_ms": per_query_ms,
        "per_query_tuning": {k: "bps%d/steal%d/split%d/flags%d" % (c["blocks_per_sm"], c["steal_interval"],
                                                                     c["min_split"], c["flags"])
                             for k, c in tuned.items()},
        "edges_visited_per_s": world * cands / (ms_per_step / 1e3),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_unit": "DRAM bytes read + written by the search kernel over one step "
                                     "(36 launches), from one ncu capture of the timed step",
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "model": "bytes_alg = 12 roots + 8 r_reads + 16 candidates of the serial "
                              "reference semantics, summed over the 36 queries"},
        "clocks": clk.summary(),
    }
    if rank == 0:
        line["c1"] = c1_leg(dev, cpu=(world == 1 and not args.no_cpu_baseline))
    if rank == 0 and world == 1 and not args.no_extra:
        line["four_cycle"] = four_cycle_leg(dg, dev, stream, flush, tune=not args.no_autotune)
        line["reference_gpu_kernel"] = ref_kernel_leg(host, dg, qs, want, dev)
        import bench_modes
        line["enumerate"] = bench_modes.enumerate_leg(warmup=1, steps=3)
        line["batch"] = bench_modes.batch_leg(window=0, n=64, limit=0, warmup=1, steps=1)
        # C5's stream shape at 2000 queries over 1000-root windows, so that the
        # one-at-a-time arm (every query exact) and the Poisson pass stay
        # within a few minutes: a handful of 5-edge queries at deltas of days
        # take seconds alone even on such windows
        line["serve"] = bench_modes.serve_leg(n=2000, window=1000, limit=int(3e7), warmup=0, steps=1)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        hi = host_info()
        threads = hi["usable_cores"]
        m, sec, kind, n = cpu_reference(args.workload, CPU_STRIDE, threads)
        m1, sec1, _, n1 = cpu_reference(args.workload, CPU_STRIDE_1T, 1)
        line["cpu_baseline"] = {
            "value": m / sec, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": cpu_sample_text(CPU_STRIDE, threads, n), "host": hi,
            "single_thread": {"value": m1 / sec1, "unit": UNIT,
                              "sample": cpu_sample_text(CPU_STRIDE_1T, 1, n1)}}
    for w in workers:
        w.close()
    dg.free()
    host.unpin()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def ref_kernel_leg(host, dg, qs, want, dev) -> dict:
    """The reference's generated search kernel (KernelGen with its warp
    options on, built for sm_100a by baseline/refgen.py) on the same 36
    queries and the same GPU, beside this library's per-query kernel.  Both
    are timed the reference's way (GPUWorker::timed_run,
    src/core/cpu/data.cc:534-542): host time around run() with the graph
    resident, best of two runs per query."""
    from baseline import refgen as R
    from everest_b200 import capi
    if not all(R.available(q["mu"], q["mv"]) for q in qs):
        return {"available": False, "why": "generated kernels not built (python -m baseline.refgen build)"}
    rg = R.RefGraph.from_host_graph(host)
    w = capi.Worker(dev)
    ref_ms, our_ms = 0.0, 0.0
    try:
        for q in qs:
            c, ms = R.count(rg, q["mu"], q["mv"], q["delta"], reps=2)
            if c != want[q["name"]]:
                raise SystemExit(f"reference kernel count mismatch on {q['name']}: {c} != {want[q['name']]}")
            ref_ms += min(ms)
            best = None
            for _ in range(2):
                w.take(dg, q["mu"], q["mv"], q["delta"])
                t0 = time.perf_counter()
                c2 = w.run()
                dt = (time.perf_counter() - t0) * 1e3
                best = dt if best is None else min(best, dt)
            if c2 != want[q["name"]]:
                raise SystemExit(f"count mismatch on {q['name']}")
            our_ms += best
    finally:
        w.close()
        rg.free()
    return {"available": True, "kernel": "reference KernelGen output (warpCentric, warpBalancing, "
                                         "tailExpansion on) for sm_100a",
            "queries": len(qs), "reference_ms": ref_ms, "this_library_ms": our_ms,
            "speedup": ref_ms / max(our_ms, 1e-9), "counts_equal": True,
            "timing": "host ms around run() per query, graph resident, best of 2; default launch parameters"}


def c1_leg(dev, cpu: bool) -> dict:
    """The CPU-runnable case: 10k nodes / 200k edges (Zipf 1.5), triangle
    0->1->2->0, delta 3600, count.  GPU: device time with the graph resident
    (best of 10 after 3 warm-up runs) and end to end from pinned host arrays
    (upload, build, query, count read back).  CPU: the reference's Baseline
    body over every root, all host cores and one thread."""
    import torch
    from everest_b200 import capi, synth
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        tri = json.load(f)["full_zipf"]["triangle"]
    spec = synth.SPECS["zipf-10k-200k"]
    u, v, t = synth.load_or_generate(spec.name)
    host = capi.graph_build_host(u, v, t, name=spec.name).pin()
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    dg = capi.DeviceGraph(host, dev, sh)
    w = capi.Worker(dev, sh)
    dev_ms = []
    for i in range(13):
        w.take(dg, tri["mu"], tri["mv"], tri["delta"])
        c = w.run()
        if c != tri["count"]:
            raise SystemExit(f"200k triangle count {c} != {tri['count']}")
        if i >= 3:
            dev_ms.append(w.last_stats()["device_ms"])
    e2e_ms = []
    for i in range(8):
        with torch.cuda.stream(stream):
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            g2 = capi.DeviceGraph(host, dev, sh)
            w.take(g2, tri["mu"], tri["mv"], tri["delta"])
            w.launch()
            c = w.result()
            ev1.record(stream)
        torch.cuda.synchronize(dev)
        g2.free()
        if c != tri["count"]:
            raise SystemExit("200k triangle end-to-end count mismatch")
        if i >= 3:
            e2e_ms.append(ev0.elapsed_time(ev1))
    w.close()
    dg.free()
    host.unpin()
    gms, ems = min(dev_ms), statistics.median(e2e_ms)
    out = {"workload": "zipf-10k-200k: 10k nodes, 200k edges, triangle 0->1->2->0, delta 3600, count",
           "count": c, "gpu_device_ms": gms, "gpu_e2e_ms": ems,
           "gpu_matches_per_s": c / (gms / 1e3), "gpu_e2e_matches_per_s": c / (ems / 1e3)}
    if cpu:
        from oracle import oracle as O
        g = O.Graph(u, v, t, spec.num_nodes)
        if O.ref_lib() is not None:
            hi = host_info()
            res = {}
            for th in (hi["usable_cores"], 1):
                best = None
                for _ in range(3):
                    t0 = time.perf_counter()
                    cc = O.ref_baseline_count(g, tri["mu"], tri["mv"], tri["delta"], threads=th)
                    dt = time.perf_counter() - t0
                    best = dt if best is None else min(best, dt)
                if cc != tri["count"]:
                    raise SystemExit("200k triangle CPU count mismatch")
                res[th] = best
            out["cpu_reference"] = {"kind": "reference", "sample": "every root", "threads": hi["usable_cores"],
                                    "ms": res[hi["usable_cores"]] * 1e3, "ms_1_thread": res[1] * 1e3,
                                    "matches_per_s": c / res[hi["usable_cores"]]}
    return out


def four_cycle_leg(dg, dev, stream, flush, tune: bool) -> dict:
    """The single-query plain kernel on a 4-edge motif: the 4-cycle
    0->1->2->3->0, delta 86400, count, on the bench graph (resident).  Device
    time of the search kernel (CUDA events on the worker's stream), L2
    flushed before every run, median of 5 after 2 warm-up runs, with the
    autotuned launch parameters (tuned outside the timing) and with the
    defaults; effective rate = the serial semantics' algorithmic bytes of
    the query (12 roots + 8 r_reads + 16 candidates, counted by the oracle)
    / kernel time, against the measured HBM copy bandwidth."""
    import torch
    from everest_b200 import autotune, capi, workloads
    st = workload_stats("bursty-7.8m-4cycle")["queries"][0]
    q = workloads.queries("bursty-7.8m-4cycle")[0]
    peak, peak_kind = measured_peaks()
    w = capi.Worker(dev, stream.cuda_stream)

    def timed(flags):
        ms = []
        for i in range(7):
            with torch.cuda.stream(stream):
                flush.zero_()
            w.take(dg, q["mu"], q["mv"], q["delta"], 0, -1, 0, flags)
            c = w.run()
            if c != st["count"]:
                raise SystemExit(f"4-cycle count {c} != {st['count']}")
            if i >= 2:
                ms.append(w.last_stats()["device_ms"])
        return statistics.median(ms)

    try:
        default_ms = timed(0)
        cfg = dict(autotune.DEFAULT)
        if tune:
            cfg = autotune.Autotuner(dev, sample_roots=0).tune(dg, q["mu"], q["mv"], q["delta"], w)
        flags = autotune.Autotuner.apply(w, cfg)
        ms = timed(flags)
    finally:
        w.close()
    ach = st["bytes_alg"] / (ms / 1e3) / 1e9
    return {"workload": "bursty-1.1m-7.8m (the bench graph): 4-cycle 0->1->2->3->0, delta 86400, count",
            "count": st["count"], "kernel_ms": ms, "kernel_ms_default_params": default_ms,
            "tuning": "bps%d/steal%d/split%d/flags%d" % (cfg["blocks_per_sm"], cfg["steal_interval"],
                                                       cfg["min_split"], cfg["flags"]),
            "bytes_alg": st["bytes_alg"], "effective_gbs": ach, "peak_gbs": peak,
            "frac": ach / peak, "peak_source": f"{peak_kind} hbm_gbs",
            "l2": "flushed before every run (256 MB write)"}


def run_single_query(args):
    """Run one query a few times on cuda:0 (for ncu captures): query I of
    the workload (--single-query), a motif on the workload's graph
    (--motif, --delta), or a constrained bench query (--constrained-query)."""
    from everest_b200 import capi, synth, workloads
    stats = workload_stats(args.workload)
    spec = synth.SPECS[stats["graph"]]
    u, v, t = synth.load_or_generate(spec.name)
    host = capi.graph_build_host(u, v, t)
    dg = capi.DeviceGraph(host, 0)
    cons = None
    if args.constrained_query:
        from everest_b200.constraints import Constraints
        byname = {name: (mu, mv, c) for name, mu, mv, c in workloads.constrained_queries()}
        mu, mv, c = byname[args.constrained_query]
        nf, ef = workloads.constrained_features(int(max(u.max(), v.max())) + 1, u.size)
        dg.set_features(nf[host.original_vertex_ids(u, v)], ef)
        q = {"name": args.constrained_query, "mu": mu, "mv": mv, "delta": c["delta"]}
        cons = Constraints.from_yaml(c, mu, mv)
    elif args.motif:
        pairs = [tuple(int(x) for x in e.split("-")) for e in args.motif.split(",")]
        q = {"name": args.motif, "mu": [a for a, b in pairs], "mv": [b for a, b in pairs], "delta": args.delta}
    else:
        q = workloads.queries(args.workload)[args.single_query]
    w = capi.Worker(0)
    for _ in range(args.reps):
        w.take(dg, q["mu"], q["mv"], q["delta"], 0, -1, 0, args.flags, constraints=cons)
        c = w.run()
        print(json.dumps({"query": q["name"], "count": c, **w.last_stats()}), flush=True)
    w.close()
    dg.free()
    return 0


def main():
    args = parse()
    if args.single_query >= 0 or args.motif or args.constrained_query:
        return run_single_query(args)
    if args.mode in ("batch", "serve", "enumerate", "constrained"):
        import bench_modes
        return bench_modes.run(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
