"""Seeded synthetic temporal graphs and motif sets for the benchmark workloads.

The public SNAP / ethereum graphs the reference was measured on are not
available offline, so every workload here is generated from a fixed seed with
``numpy.random.Generator(PCG64(seed))``.  The generated edge list is already
in the order the reference's loader produces (stable sort by timestamp,
``src/core/cpu/data.cc:246-248``): edges are sorted by ``(t, draw index)``, so
the edge id equals the line index and the original-line index (``Euid``) is
the identity.

Graph families
--------------
``zipf``   (the 200k-edge CPU-runnable case): ``src`` and ``dst`` are drawn
           independently from a bounded Zipf(s) law over ranks ``1..V``, mapped
           to node ids through one seeded permutation; pairs with
           ``src == dst`` are redrawn; timestamps are uniform in ``[0, t_max)``.
``bursty`` (the 7.8M / 36M / 63M-edge cases): node activity comes in bursts.
           A burst picks one source node with probability proportional to a
           discrete Pareto weight ``rank**(-1/(alpha-1))`` (so out-degrees
           follow a power law with exponent ``alpha``), a start time uniform
           in ``[0, t_span)``, a size ``max(1, Poisson(burst_mean))`` and
           exponential inter-edge gaps of mean ``gap_mean`` seconds.  Each
           edge of the burst draws its destination independently from a power
           law over the same node ranking (nodes that send much also receive
           much, as in message graphs); a destination equal to the source is
           redrawn.  With probability ``reply`` an edge after the first is a
           reply instead: it goes from the destination of the burst's latest
           non-reply edge back to the burst's source.  Bursts are generated until ``E`` edges
           exist, then truncated to exactly ``E``.
"""
from __future__ import annotations

import dataclasses
import json
import os
from typing import Dict, List, Tuple

import numpy as np

__all__ = [
    "GraphSpec", "SPECS", "generate", "load_or_generate", "write_edge_text",
    "three_edge_patterns", "random_patterns", "motif_text",
]


@dataclasses.dataclass(frozen=True)
class GraphSpec:
    name: str
    family: str          # "zipf" | "bursty"
    num_nodes: int
    num_edges: int
    seed: int
    zipf_s: float = 1.5          # zipf family
    t_max: int = 10_000_000      # zipf family: t ~ U{0..t_max-1}
    alpha: float = 2.1           # bursty family: power-law degree exponent
    t_span: int = 230_000_000    # bursty family: burst starts ~ U[0, t_span)
    burst_mean: float = 20.0     # bursty family: Poisson mean burst size
    gap_mean: float = 60.0       # bursty family: mean intra-burst gap (s)
    reply: float = 0.25          # bursty family: probability an edge answers the burst source


SPECS: Dict[str, GraphSpec] = {
    # 10k nodes / 200k edges, zipf 1.5, uniform t in [0, 1e7)
    "zipf-10k-200k": GraphSpec("zipf-10k-200k", "zipf", 10_000, 200_000, seed=1),
    # 1.1M nodes / 7.8M edges, power law 2.1, bursty over 2.3e8 s
    "bursty-1.1m-7.8m": GraphSpec("bursty-1.1m-7.8m", "bursty", 1_100_000, 7_800_000, seed=2),
    # 2.6M nodes / 36M edges, same generator
    "bursty-2.6m-36m": GraphSpec("bursty-2.6m-36m", "bursty", 2_600_000, 36_000_000, seed=3),
    # 6M nodes / 63M edges, same generator
    "bursty-6m-63m": GraphSpec("bursty-6m-63m", "bursty", 6_000_000, 63_000_000, seed=5),
}


def _zipf_sampler(rng: np.random.Generator, n: int, s: float):
    w = np.arange(1, n + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]

    def draw(size: int) -> np.ndarray:
        r = np.searchsorted(cdf, rng.random(size), side="right")
        return np.minimum(r, n - 1).astype(np.int64)
    return draw


def _gen_zipf(spec: GraphSpec, rng: np.random.Generator):
    V, E = spec.num_nodes, spec.num_edges
    perm = rng.permutation(V).astype(np.int32)
    draw = _zipf_sampler(rng, V, spec.zipf_s)
    src = draw(E)
    dst = draw(E)
    bad = src == dst
    while bad.any():
        k = int(bad.sum())
        src[bad] = draw(k)
        dst[bad] = draw(k)
        bad = src == dst
    t = rng.integers(0, spec.t_max, size=E, dtype=np.int64)
    return perm[src], perm[dst], t


def _gen_bursty(spec: GraphSpec, rng: np.random.Generator):
    V, E = spec.num_nodes, spec.num_edges
    s = 1.0 / (spec.alpha - 1.0)
    perm = rng.permutation(V).astype(np.int32)
    draw_src = _zipf_sampler(rng, V, s)
    draw_dst = _zipf_sampler(rng, V, s)
    # enough bursts for E edges (mean size >= burst_mean for Poisson clipped at 1)
    nb = int(E / spec.burst_mean * 1.05) + 16
    sizes = np.maximum(1, rng.poisson(spec.burst_mean, size=nb))
    while sizes.sum() < E:
        extra = np.maximum(1, rng.poisson(spec.burst_mean, size=nb // 10 + 16))
        sizes = np.concatenate([sizes, extra])
    csum = np.cumsum(sizes)
    nb = int(np.searchsorted(csum, E, side="left")) + 1
    sizes = sizes[:nb].copy()
    sizes[-1] -= int(csum[nb - 1] - E)
    starts = rng.random(nb) * spec.t_span
    burst_src = draw_src(nb)
    burst_of = np.repeat(np.arange(nb, dtype=np.int64), sizes)
    gaps = rng.exponential(spec.gap_mean, size=E)
    # time of an edge = burst start + cumulative gaps inside its burst
    first = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    cg = np.cumsum(gaps)
    base = cg[first] - gaps[first]           # cumulative gap before the burst's first edge
    t = np.floor(starts[burst_of] + (cg - base[burst_of])).astype(np.int64)
    s_ids = perm[burst_src[burst_of]]
    d_ids = perm[draw_dst(E)]
    bad = s_ids == d_ids
    while bad.any():
        k = int(bad.sum())
        d_ids[bad] = perm[draw_dst(k)]
        bad = s_ids == d_ids
    # replies: edge i (not the first of its burst) answers the burst source
    # from the destination of the burst's latest non-reply edge
    idx = np.arange(E, dtype=np.int64)
    pos_in_burst = idx - first[burst_of]
    rep = (rng.random(E) < spec.reply) & (pos_in_burst > 0)
    last_plain = np.maximum.accumulate(np.where(rep, -1, idx))  # first edge of a burst is plain
    src_out, dst_out = s_ids.copy(), d_ids.copy()
    src_out[rep] = d_ids[last_plain[rep]]
    dst_out[rep] = s_ids[rep]
    return src_out, dst_out, t


def generate(spec: GraphSpec) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Return ``(u, v, t)`` int32 arrays sorted by ``(t, draw index)``."""
    rng = np.random.Generator(np.random.PCG64(spec.seed))
    if spec.family == "zipf":
        u, v, t = _gen_zipf(spec, rng)
    elif spec.family == "bursty":
        u, v, t = _gen_bursty(spec, rng)
    else:
        raise ValueError(f"unknown family {spec.family}")
    order = np.argsort(t, kind="stable")
    t = t[order]
    if t.size and (t.min() < 0 or t.max() > np.iinfo(np.int32).max):
        raise OverflowError("timestamps do not fit int32")
    return (np.ascontiguousarray(u[order], dtype=np.int32),
            np.ascontiguousarray(v[order], dtype=np.int32),
            np.ascontiguousarray(t, dtype=np.int32))


def data_dir() -> str:
    d = os.environ.get("EVX_DATA_DIR") or os.path.join(
        os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "_data")
    os.makedirs(d, exist_ok=True)
    return d


def load_or_generate(name: str):
    """Generate (or load from ``_data/<name>.npz``) the named graph."""
    spec = SPECS[name]
    path = os.path.join(data_dir(), f"{name}.npz")
    if os.path.exists(path):
        z = np.load(path)
        if json.loads(str(z["spec"])) == dataclasses.asdict(spec):
            return z["u"], z["v"], z["t"]
    u, v, t = generate(spec)
    tmp = path + f".tmp{os.getpid()}.npz"
    np.savez(tmp, u=u, v=v, t=t, spec=json.dumps(dataclasses.asdict(spec)))
    os.replace(tmp, path)
    return u, v, t


def write_edge_text(path: str, u: np.ndarray, v: np.ndarray, t: np.ndarray) -> None:
    """Write ``u v t`` lines (the reference's graph text format)."""
    arr = np.stack([u, v, t], axis=1)
    np.savetxt(path, arr, fmt="%d")


# ---------------------------------------------------------------- motifs ----

def three_edge_patterns() -> List[List[Tuple[int, int]]]:
    """All connected 3-edge temporal patterns on 2..3 nodes, by rule.

    Rule: the first edge is ``0->1``; every later edge touches an already
    mapped node; a new node takes the next id; no self-loops.  This is the
    reference's own motif precondition (``HostMotifData``,
    ``src/core/cpu/data.cc:411-449``) and yields 36 patterns.
    """
    out = []

    def rec(edges, nn):
        if len(edges) == 3:
            out.append(list(edges))
            return
        cands = []
        for a in range(nn + 1):
            for b in range(nn + 1):
                if a == b:
                    continue
                if a == nn and b == nn:
                    continue
                if a == nn or b == nn:
                    if nn >= 3:
                        continue
                cands.append((a, b))
        for a, b in cands:
            rec(edges + [(a, b)], max(nn, a + 1, b + 1))
    rec([(0, 1)], 2)
    return out


def random_patterns(count: int, edge_range, node_range, seed: int):
    """Random connected patterns (same rule), ``k`` edges and ``n`` nodes drawn
    uniformly from the inclusive ranges; patterns are deduplicated."""
    rng = np.random.Generator(np.random.PCG64(seed))
    seen, out = set(), []
    tries = 0
    while len(out) < count:
        tries += 1
        if tries > 1000 * count:
            raise RuntimeError("cannot draw enough distinct patterns")
        k = int(rng.integers(edge_range[0], edge_range[1] + 1))
        n = int(rng.integers(node_range[0], node_range[1] + 1))
        if n > k + 1 or (n == 2 and k < 1):
            continue
        edges, nn = [(0, 1)], 2
        ok = True
        for j in range(1, k):
            remaining = k - j
            need_new = n - nn
            if need_new > remaining:
                ok = False
                break
            must_new = need_new == remaining
            can_new = need_new > 0
            new = must_new or (can_new and rng.random() < 0.5)
            if new:
                a = int(rng.integers(0, nn))
                if rng.random() < 0.5:
                    edges.append((a, nn))
                else:
                    edges.append((nn, a))
                nn += 1
            else:
                if nn < 2:
                    ok = False
                    break
                a, b = rng.choice(nn, size=2, replace=False)
                edges.append((int(a), int(b)))
        if not ok or nn != n:
            continue
        key = tuple(edges)
        if key in seen:
            continue
        seen.add(key)
        out.append(edges)
    return out


def motif_text(edges) -> str:
    """Motif file text (``u v t`` per line, 1-based node labels like the
    reference's ``inputs/motifs/*.txt``)."""
    return "".join(f"{a + 1} {b + 1} {i + 1}\n" for i, (a, b) in enumerate(edges))
