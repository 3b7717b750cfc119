"""Batched and served query throughput against one-at-a-time plain kernels
(``bench.py --mode batch`` / ``--mode serve``).

batch: 64 mixed 3/4-edge queries on the 36M-edge graph
    (``workloads.batch_queries``) in one persistent launch replayed from a
    CUDA graph, against the same queries run one at a time through the
    per-query kernel (evx_worker_take + evx_worker_run each).
serve: a stream of 3-5-edge count and enumerate queries on two resident
    graphs (7.8M and 63M edges; ``workloads.serve_queries``) through
    ``serve.Server``, against the same queries one at a time.  Reported:
    queries/s with every query submitted at once (saturation; the median of
    --steps runs, each listed), and latency
    percentiles under a Poisson arrival stream at 0.8x the one-at-a-time
    capacity.  The one-at-a-time server's latency under the same arrival
    times is that of a FIFO single server with the measured service times.

Both arms apply the same work limit per query (adjacency records examined
inside their time windows); a query past it is stopped and flagged in both
(the flag depends only on the graph and the query).  Every other result must
be equal in both arms, and is checked.
"""
from __future__ import annotations

import json
import os
import time
from typing import Dict, List

import numpy as np


def _one_at_a_time(capi, dgs: Dict[str, object], qs: List[dict], limit: int):
    """Run each query alone through the per-query kernel; returns per-query
    (count, limited, rows_or_None) and service seconds."""
    w = capi.Worker(0)
    w.set_limit(limit)
    res, svc = [], []
    for q in qs:
        s0 = time.perf_counter()
        w.take(dgs[q["graph"]], q["mu"], q["mv"], q["delta"], q["beg"], q["end"], q["cap"])
        limited = False
        try:
            c = w.run()
        except capi.LimitExceeded as e:
            c, limited = e.count, True
        rows = w.enum_rows(q["cap"]) if q["cap"] else None
        svc.append(time.perf_counter() - s0)
        res.append((c, limited, rows))
    w.close()
    return res, np.array(svc)


def _same(a, b, q) -> bool:
    """Equal results: exact counts equal, limited flags equal; enumerations
    below their cap equal as row sets, capped ones both at the cap."""
    (ca, la, ra), (cb, lb, rb) = a, b
    if la or lb:
        return la and lb
    if q["cap"] and (ca > q["cap"] or cb > q["cap"]):
        return ca >= q["cap"] and cb >= q["cap"] and len(ra) == len(rb) == q["cap"]
    if ca != cb:
        return False
    if q["cap"]:
        return sorted(map(tuple, ra.tolist())) == sorted(map(tuple, rb.tolist()))
    return True


def _pct(x, p):
    return float(np.percentile(np.asarray(x) * 1e3, p))


def batch_leg(window: int = 0, n: int = 64, limit: int = 0, warmup: int = 1, steps: int = 1,
              tune: bool = False, tile: int = 64) -> dict:
    """C3: n random connected 3/4-edge patterns on 2-4 nodes, delta cycling
    3600 / 86400 / 604800, on the 2.6M-node / 36M-edge graph, in one
    persistent launch per motif size replayed from a CUDA graph, against the
    same queries one at a time through the per-query kernel
    (evx_worker_take + evx_worker_run each).  window = 0: every root of the
    graph (C3 as specified); else a random window of that many roots per
    query.  limit = 0: every result exact; else queries past the limit are
    flagged in both arms.  Results are checked equal."""
    import torch
    from everest_b200 import autotune, capi, synth, workloads
    torch.cuda.set_device(0)
    qs = workloads.batch_queries(window or 1_000_000, n)
    if not window:
        qs = [dict(q, beg=0, end=-1) for q in qs]
    spec = synth.SPECS["bursty-2.6m-36m"]
    u, v, t = synth.load_or_generate(spec.name)
    dg = capi.DeviceGraph(capi.graph_build_host(u, v, t, name=spec.name), 0)
    dgs = {spec.name: dg}
    seq_s, svc_all = [], None
    for rep in range(warmup + steps):
        res, svc = _one_at_a_time(capi, dgs, qs, limit)
        if rep >= warmup:
            seq_s.append(float(svc.sum()))
            svc_all = svc
    seq = res
    tq = [(q["mu"], q["mv"], q["delta"], q["beg"], q["end"]) for q in qs]
    if tune:
        tile = autotune.Autotuner(0).tune_batch(lambda: capi.Batch(0, max(64, n)), tq, dg, limit=limit)
    b = capi.Batch(0, max(64, n))
    b.set_tuning(tile_roots=tile)
    if limit:
        b.set_limit(limit)
    for q in tq:
        b.add(dg, *q)
    bat_s, dev_ms = [], []
    for rep in range(warmup + steps):
        t0 = time.perf_counter()
        r = b.run()
        dt = time.perf_counter() - t0
        if rep >= warmup:
            bat_s.append(dt)
            dev_ms.append(b.last_stats()["device_ms"])
    b.close()
    dg.free()
    bat = [(c, c == capi.LIMITED, None) for c in r]
    bad = [i for i, q in enumerate(qs) if not _same(seq[i], bat[i], q)]
    if bad:
        raise SystemExit(f"batched results differ from one-at-a-time results for queries {bad[:8]}")
    t_seq = float(np.mean(seq_s))
    t_bat = float(np.mean(bat_s))
    order = np.argsort(-svc_all)
    top5 = float(svc_all[order[:5]].sum())
    heavy = [[int(i), "".join(f"{a}{b_}" for a, b_ in zip(qs[i]["mu"], qs[i]["mv"])), qs[i]["delta"],
              round(float(svc_all[i]) * 1e3, 1)] for i in order[:5]]
    why = (f"the five heaviest queries take {100 * top5 / max(float(svc_all.sum()), 1e-12):.0f} % of the "
           "one-at-a-time time and each already fills the GPU on its own; batching saves only per-query "
           "launch, synchronisation and tail time, which the light queries "
           f"({int((svc_all < 0.02).sum())} under 20 ms) add up to little of")
    return {"metric": "batched queries/s (one persistent launch per motif size) vs one at a time, exact",
            "value": n / t_bat, "unit": "queries/s", "ms": t_bat * 1e3, "steps": steps, "warmup": warmup,
            "config": {"workload": f"bursty 2.6M nodes / 36M edges; {n} random connected 3/4-edge patterns "
                                   "on 2-4 nodes, delta cycling 3600/86400/604800, " +
                                   (f"roots = a random window of {window} edges per query" if window
                                    else "every root of the graph"),
                       "tile_roots": tile, "work_limit": limit or None, "cuda_graph": True},
            "one_at_a_time": {"value": n / t_seq, "unit": "queries/s", "ms": t_seq * 1e3,
                              "heaviest_ms": heavy},
            "speedup": t_seq / t_bat, "batched_device_ms": float(np.mean(dev_ms)),
            "matches": int(sum(c for c, lim, _ in seq if not lim)),
            "limited_queries": int(sum(lim for _, lim, _ in seq)), "results_equal": True,
            "why_not_3x": why if t_seq / t_bat < 3 else None}


def run_batch(args) -> int:
    """``bench.py --mode batch``: batch_leg as its own JSON line (--window 0:
    the whole graph; --limit 0: exact)."""
    leg = batch_leg(window=args.window, n=args.queries or 64, limit=int(args.limit or 0), warmup=args.warmup,
                    steps=args.steps, tune=True)
    line = {"metric": leg["metric"], "value": leg["value"], "unit": "queries/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": leg["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator)", "mode": "batch"}
    line.update({k: v for k, v in leg.items() if k not in ("metric", "value", "unit", "ms")})
    print(json.dumps(line), flush=True)
    return 0


def serve_leg(n: int = 10_000, window: int = 100_000, limit: int = int(3e7), warmup: int = 1, steps: int = 3,
              slots: str = "64,2,2,2,1.0,2,2") -> dict:
    """Serving: a stream of n 3-5-edge count and enumerate queries on two
    resident graphs (7.8M and 63M edges; ``workloads.serve_queries``)
    through ``serve.Server``, against the same queries one at a time through
    the plain per-query kernel, every result exact in both (checked).

    The one-at-a-time arm runs each query alone with no work limit; its
    service times give its capacity and, under the Poisson arrival times
    below, the latency of a FIFO server.  The served arm keeps queries past
    ``limit`` adjacency records out of the shared batches and re-runs them
    on heavy slots (no limit, a fraction of the SMs beside other work).
    Reported: queries/s with every query submitted at once (the median of
    ``steps`` passes after ``warmup``), and p50 / p99 / p99.9 latency under
    Poisson arrivals at 0.8x the one-at-a-time capacity, beside FIFO's."""
    import torch
    from everest_b200 import capi, serve, synth, workloads
    torch.cuda.set_device(0)
    qs = workloads.serve_queries(window, n)
    hosts = {}
    for key in ("bursty-1.1m-7.8m", "bursty-6m-63m"):
        sp = synth.SPECS[key]
        u, v, t = synth.load_or_generate(sp.name)
        hosts[sp.name] = capi.graph_build_host(u, v, t, name=sp.name)
    dgs = {k: capi.DeviceGraph(h, 0) for k, h in hosts.items()}
    _one_at_a_time(capi, dgs, qs[: min(64, n)], 0)  # warm-up
    seq, svc = _one_at_a_time(capi, dgs, qs, 0)
    for g in dgs.values():
        g.free()
    seq_total = float(svc.sum())
    seq_qps = n / seq_total
    rate = 0.8 * seq_qps
    arr = np.cumsum(np.random.Generator(np.random.PCG64(11)).exponential(1.0 / rate, size=n))
    # the one-at-a-time server under those arrivals: FIFO, one query at a time
    fin = np.empty(n)
    prev = 0.0
    for i in range(n):
        prev = max(arr[i], prev) + svc[i]
        fin[i] = prev
    seq_lat = fin - arr
    out = {}
    sl = [float(x) for x in slots.split(",")]
    sl += [64, 2, 2, 2, 1.0, 2, 2][len(sl):]
    mb, ib, es, ebps = (int(x) for x in sl[:4])
    share = sl[4]
    hs, hbps = int(sl[5]), int(sl[6])
    runs = [("warmup", None)] * max(0, warmup) + [("saturated", None)] * max(1, steps) + [("poisson", arr)]
    sat_runs = []
    for label, times in runs:
        srv = serve.Server(0, max_batch=mb, inflight_batches=ib, enum_slots=es, limit=limit,
                           enum_blocks_per_sm=ebps, batch_share=share, heavy_slots=hs,
                           heavy_blocks_per_sm=hbps)
        for k, h in hosts.items():
            srv.add_graph(k, h)
        futs = []
        t0 = time.perf_counter()
        for i, q in enumerate(qs):
            if times is not None:
                d = t0 + times[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
            futs.append(srv.submit(q["graph"], q["mu"], q["mv"], q["delta"], q["cap"], 0, q["beg"], q["end"]))
        srv.drain(3600)
        got = [f.result() for f in futs]
        served = [(r.count, r.limited, r.rows) for r in got]
        bad = [i for i, q in enumerate(qs) if not _same(seq[i], served[i], q)]
        if bad:
            raise SystemExit(f"served results differ from one-at-a-time results for queries {bad[:8]}")
        st = srv.stats()
        st["unanswered"] = sum(1 for r in got if r.count is None)
        if label == "saturated":
            sat_runs.append(st)
        elif label == "poisson":
            out[label] = st
        srv.close()
    sat_runs.sort(key=lambda x: x["queries_per_s"])
    out["saturated"] = dict(sat_runs[len(sat_runs) // 2])
    out["saturated"]["runs_queries_per_s"] = [round(x["queries_per_s"], 1) for x in sat_runs]
    cnt = [i for i, q in enumerate(qs) if not q["cap"]]
    order = np.argsort(-svc)
    top = float(svc[order[:10]].sum())
    speedup = out["saturated"]["queries_per_s"] / seq_qps
    why = None
    if speedup < 3:
        why = (f"the ten heaviest queries take {100 * top / max(seq_total, 1e-12):.0f} % of the one-at-a-time "
               f"time (the longest alone {1e3 * float(svc[order[0]]):.0f} ms, a 5-edge motif over a hub's "
               "window); each fills the GPU on its own and its work is in a few roots, so serving can only "
               "overlap the rest with it: the served makespan is bounded below by the heaviest query")
    return {
        "metric": "served queries/s and p50/p99/p99.9 latency vs one at a time, exact",
        "value": out["saturated"]["queries_per_s"], "unit": "queries/s",
        "config": {"workload": f"bursty 7.8M + 63M edges resident; {n} queries, 3-5-edge patterns on 2-4 "
                               "nodes, delta log-uniform [600, 604800], 20% enumerate (cap log-uniform "
                               f"[1e4, 1e6]), roots = a random window of {window} edges per query",
                   "batch_work_limit": limit, "poisson_rate_qps": rate,
                   "max_batch": mb, "batches_in_flight": ib, "enumeration_slots": es,
                   "enumeration_blocks_per_sm": ebps, "batch_share": share, "heavy_slots": hs,
                   "heavy_blocks_per_sm": hbps, "warmup": warmup, "steps": steps},
        "one_at_a_time": {"value": seq_qps, "unit": "queries/s", "work_limit": None,
                          "service_s": {"count": float(sum(svc[i] for i in cnt)),
                                        "enumerate": float(sum(svc[i] for i, q in enumerate(qs) if q["cap"]))},
                          "service_p50_ms": _pct(svc, 50), "service_p99_ms": _pct(svc, 99),
                          "longest_ms": sorted(([int(i), round(float(svc[i]) * 1e3, 2), len(qs[i]["mu"]),
                                                 qs[i]["cap"]] for i in range(n)), key=lambda x: -x[1])[:5],
                          "poisson_p50_ms": _pct(seq_lat, 50), "poisson_p99_ms": _pct(seq_lat, 99),
                          "poisson_p999_ms": _pct(seq_lat, 99.9)},
        "served_saturated": out["saturated"], "served_poisson_0.8x": out["poisson"],
        "speedup": speedup, "why_not_3x": why,
        "p99_vs_fifo": out["poisson"]["p99_ms"] / max(_pct(seq_lat, 99), 1e-9),
        "count_queries": len(cnt), "enumerate_queries": n - len(cnt),
        "requeued_queries": out["saturated"]["requeued"],
        "limited_unanswered": out["saturated"]["unanswered"] + out["poisson"]["unanswered"],
        "results_equal": True}


def run_serve(args) -> int:
    """``bench.py --mode serve``: serve_leg as its own JSON line."""
    leg = serve_leg(n=args.queries or 10_000, window=args.window or 100_000,
                    limit=int(args.limit if args.limit is not None else 3e7),
                    warmup=args.warmup, steps=args.steps, slots=getattr(args, "serve_slots", "64,2,2,2,1.0,2,2"))
    line = {"metric": leg["metric"], "value": leg["value"], "unit": "queries/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * (args.queries or 10_000) / max(leg["value"], 1e-9), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator)",
            "mode": "serve"}
    line.update({k: v for k, v in leg.items() if k not in ("metric", "value", "unit")})
    print(json.dumps(line), flush=True)
    return 0


def full_size_counts() -> dict:
    """Counts at full size from the reference's generated kernel on a B200
    (tests/golden/full_size_counts.json, written by
    tests/golden/make_full_size_counts.py)."""
    p = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "full_size_counts.json")
    with open(p) as f:
        return json.load(f)


def enumerate_leg(warmup: int = 3, steps: int = 5) -> dict:
    """Enumeration under memory admission: the 4-cycle 0->1->2->3->0 on the
    2.6M-node / 36M-edge graph, delta 86400, cap 1e6.  The row buffer
    (cap x 4 int32) is admitted against free device memory by the worker.
    Reported: rows/s of the capped enumeration, the exact total count (equal
    to the reference's generated kernel's) and its time, and a host check
    that every returned row is a distinct valid match (edge order, window,
    endpoints, injectivity)."""
    import torch
    from everest_b200 import capi, synth
    torch.cuda.set_device(0)
    spec = synth.SPECS["bursty-2.6m-36m"]
    u, v, t = synth.load_or_generate(spec.name)
    dg = capi.DeviceGraph(capi.graph_build_host(u, v, t, name=spec.name), 0)
    mu, mv, delta, cap = [0, 1, 2, 3], [1, 2, 3, 0], 86400, 1_000_000
    w = capi.Worker(0)
    count_ms, enum_ms = [], []
    total = rows = None
    for rep in range(warmup + steps):
        w.take(dg, mu, mv, delta)
        total = w.run()
        cm = w.last_stats()["device_ms"]
        w.take(dg, mu, mv, delta, 0, -1, cap)
        w.run()
        em = w.last_stats()["device_ms"]
        rows = w.enum_rows(cap)
        if rep >= warmup:
            count_ms.append(cm)
            enum_ms.append(em)
    w.close()
    dg.free()
    want = full_size_counts()["bursty-2.6m-36m"]["4-cycle delta 86400"]
    if total != want:
        raise SystemExit(f"4-cycle total {total} != the reference kernel's {want}")
    # host validation of the rows (line ids = sorted edge ids for this graph)
    r = rows.astype(np.int64)
    ok = (r[:, 0] < r[:, 1]) & (r[:, 1] < r[:, 2]) & (r[:, 2] < r[:, 3])
    ok &= t[r[:, 3]] <= t[r[:, 0]] + delta
    a, b = u[r[:, 0]], v[r[:, 0]]
    ok &= (u[r[:, 1]] == b) & (u[r[:, 2]] == v[r[:, 1]]) & (u[r[:, 3]] == v[r[:, 2]]) & (v[r[:, 3]] == a)
    c_, d_ = v[r[:, 1]], v[r[:, 2]]
    ok &= (a != b) & (a != c_) & (a != d_) & (b != c_) & (b != d_) & (c_ != d_)
    distinct = len(np.unique(r, axis=0)) == len(r)
    n_rows = int(len(rows))
    expect_rows = min(cap, total)
    if not (ok.all() and distinct and n_rows == expect_rows):
        raise SystemExit("enumeration rows failed the host check")
    em = float(np.median(enum_ms))
    return {"metric": "enumerated rows/s under memory admission (capped), exact total beside it",
            "value": n_rows / (em / 1e3), "unit": "rows/s", "ms": em, "steps": steps, "warmup": warmup,
            "config": {"workload": "bursty 2.6M nodes / 36M edges; 4-cycle 0->1->2->3->0, delta 86400, "
                                   "enumerate cap 1e6 (int32 rows of original line ids)",
                       "row_buffer_bytes": cap * 4 * 4},
            "rows": n_rows, "exact_total": int(total), "exact_total_equals_reference_kernel": True,
            "count_ms": float(np.median(count_ms)), "rows_valid_distinct": True}


def run_enumerate(args) -> int:
    """``bench.py --mode enumerate``: enumerate_leg as its own JSON line."""
    leg = enumerate_leg(args.warmup, args.steps)
    line = {"metric": leg["metric"], "value": leg["value"], "unit": "rows/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": leg["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator)", "mode": "enumerate",
            "config": leg["config"], "rows": leg["rows"], "exact_total": leg["exact_total"],
            "count_ms": leg["count_ms"], "rows_valid_distinct": True}
    print(json.dumps(line), flush=True)
    return 0


def constrained_cpu(u, v, t, queries, nf, ef) -> List[dict]:
    """The host side of ``--mode constrained``: each query's count and time
    on all host cores, through the reference's own generated search (the
    KernelGen body built for the host, oracle/_ref/gen_<name>.so, where the
    build had the reference tree) and through the oracle."""
    from oracle import oracle as O
    from oracle import ref_generated as RG
    from everest_b200.constraints import Constraints
    V = int(max(u.max(), v.max())) + 1
    g = O.Graph(u, v, t, V)
    out = []
    for name, mu, mv, cons in queries:
        c = Constraints.from_yaml(cons, mu, mv)
        t0 = time.perf_counter()
        oracle_count = O.count_constrained(g, mu, mv, cons["delta"], c.to_struct(), nf, ef)
        row = {"query": name, "oracle_count": oracle_count, "oracle_ms": (time.perf_counter() - t0) * 1e3}
        so = RG.bench_library(name)
        if os.path.exists(so):
            t0 = time.perf_counter()
            row["reference_count"] = RG.GeneratedSearch(so).run(g, nf, ef, mu, mv, cons["delta"])
            row["reference_ms"] = (time.perf_counter() - t0) * 1e3
        out.append(row)
    return out


def run_constrained(args) -> int:
    """Constrained queries (``workloads.constrained_queries``: the shapes of
    the reference's additional-features query set, node predicates, temporal
    gaps, an anti-edge and a filter) on the 7.8M-edge graph with seeded node
    and edge features uniform in [0, 1e9) (the reference draws them from a
    file of random integers in that range).  Reported per query: the search
    kernel's device time and the count, checked against the reference's own
    generated search built for the host (where present) and the oracle, with
    their times on all host cores; the reference's is the cpu_baseline."""
    import torch
    from everest_b200 import capi, synth, workloads
    from everest_b200.constraints import Constraints
    torch.cuda.set_device(0)
    spec = synth.SPECS["bursty-1.1m-7.8m"]
    u, v, t = synth.load_or_generate(spec.name)
    host = capi.graph_build_host(u, v, t, name=spec.name)
    dg = capi.DeviceGraph(host, 0)
    V = int(max(u.max(), v.max())) + 1
    nf, ef = workloads.constrained_features(V, u.size)
    dg.set_features(nf[host.original_vertex_ids(u, v)], ef)
    queries = workloads.constrained_queries()
    w = capi.Worker(0)
    out = []
    for name, mu, mv, cons in queries:
        c = Constraints.from_yaml(cons, mu, mv)
        ms = []
        count = None
        for rep in range(args.warmup + args.steps):
            w.take(dg, mu, mv, cons["delta"], constraints=c)
            count = w.run()
            if rep >= args.warmup:
                ms.append(w.last_stats()["device_ms"])
        out.append({"query": name, "count": int(count), "search_ms": float(np.median(ms))})
    mu, mv = queries[0][1], queries[0][2]
    w.take(dg, mu, mv, queries[0][3]["delta"])
    plain = w.run()
    w.close()
    dg.free()
    cpu = constrained_cpu(u, v, t, queries, nf, ef)
    ok = int(plain) == out[0]["count"]
    for q, c in zip(out, cpu):
        q["oracle_equal"] = q["count"] == c["oracle_count"]
        q["oracle_ms_all_cores"] = c["oracle_ms"]
        ok &= q["oracle_equal"]
        if "reference_count" in c:
            q["reference_equal"] = q["count"] == c["reference_count"]
            q["reference_ms_all_cores"] = c["reference_ms"]
            ok &= q["reference_equal"]
    ref = all("reference_ms" in c for c in cpu)
    cpu_ms = sum(c["reference_ms" if ref else "oracle_ms"] for c in cpu)
    tot_ms = sum(q["search_ms"] for q in out)
    line = {"metric": "constrained queries/s (reference additional-features query shapes)",
            "value": len(out) / (tot_ms / 1e3), "unit": "queries/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator and features)",
            "mode": "constrained",
            "config": {"workload": "bursty 1.1M nodes / 7.8M edges, node and edge features U[0, 1e9); "
                                   "4-cycle and 4-cycle with anti-edge, delta 86400, gaps 21600 / 43200"},
            "queries": out, "plain_kernel_M4_count": int(plain),
            "cpu_baseline": {"value": len(out) / (cpu_ms / 1e3), "unit": "queries/s", "cores": os.cpu_count(),
                             "kind": "reference" if ref else "port",
                             "sample": "the same five queries, whole graph" +
                                       (" (the reference's generated search body built for the host)" if ref
                                        else " (the oracle)")},
            "all_counts_equal": bool(ok)}
    print(json.dumps(line), flush=True)
    return 0 if ok else 1


def run(args) -> int:
    if args.mode == "batch":
        return run_batch(args)
    if args.mode == "enumerate":
        return run_enumerate(args)
    if args.mode == "constrained":
        return run_constrained(args)
    return run_serve(args)
