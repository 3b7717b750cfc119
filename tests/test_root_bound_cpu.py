"""The invariant behind the search kernel's per-root window bound, checked on
the host against brute force (no GPU).

When the last motif edge has root node 0 or 1 as its target (source), every
match's last edge lies in that graph node's in-list (out-list) after the root
edge and inside the window t(e_0) + delta.  So every edge of a match is at
most L, the last such entry (edges are time-sorted: a smaller id never has a
later timestamp), and a root with no such entry has no match.  The kernel
drops those roots and ends each other root's window at t(L); these tests
check, for random tiny graphs and motifs of 3-5 edges, that every
brute-force match satisfies the bound and that no dropped root has one."""
import numpy as np

from everest_b200 import synth
from oracle import oracle as O


def _bound(u, v, t, mu, mv, delta, e0):
    """(side, L) for root e0: side -1 when the last edge touches neither root
    node (no bound), L = -1 when the bounding list has no entry."""
    a, b = mu[-1], mv[-1]
    if b <= 1:
        x, col = (u[e0] if b == 0 else v[e0]), v  # in-list of x: edges whose target is x
    elif a <= 1:
        x, col = (u[e0] if a == 0 else v[e0]), u  # out-list of x: edges whose source is x
    else:
        return -1, None
    tl = int(t[e0]) + delta
    cand = [e for e in range(e0 + 1, len(u)) if col[e] == x and int(t[e]) <= tl]
    return 0, (cand[-1] if cand else -1)


def test_window_bound_holds_for_every_match():
    rng = np.random.default_rng(2024)
    checked = dropped = 0
    for trial in range(200):
        E = int(rng.integers(8, 24))
        V = int(rng.integers(2, 5))
        u = rng.integers(0, V, E).astype(np.int32)
        v = rng.integers(0, V, E).astype(np.int32)
        t = np.sort(rng.integers(0, 12, E)).astype(np.int32)
        k = int(rng.integers(3, 6))
        pat = synth.random_patterns(1, (k, k), (2, min(k + 1, 5)), seed=trial)[0]
        mu, mv = [a for a, b in pat], [b for a, b in pat]
        delta = int(rng.integers(2, 12))
        rows = O.brute_force(u, v, t, mu, mv, delta)
        by_root = {}
        for r in rows:
            by_root.setdefault(r[0], []).append(r)
        for e0 in range(E):
            if u[e0] == v[e0]:
                continue
            side, L = _bound(u, v, t, mu, mv, delta, e0)
            if side < 0:
                continue
            if L < 0:
                assert e0 not in by_root, (trial, mu, mv, delta, e0)  # a dropped root has no match
                dropped += 1
                continue
            for r in by_root.get(e0, []):
                assert max(r) <= L, (trial, mu, mv, delta, r, L)
                assert all(int(t[e]) <= int(t[L]) for e in r)
                checked += 1
    assert checked > 150 and dropped > 150, (checked, dropped)
