// Per-motif backtracking search for temporal motifs on sm_100a.
//
// Semantics (bit-exact with the reference's generated kernel,
// system/templates/dispatch/top.snp and system/templates/common/*.snp):
// a match is a tuple of edge ids e_0 < e_1 < ... < e_{k-1} with
// u(e_0) != v(e_0), t(e_j) <= t(e_0) + delta, and an injective map of motif
// nodes to graph nodes.  Motif edge j >= 1 is searched in the out-list of the
// image of its source when its target is new, the in-list of the image of its
// target when its source is new, and the shorter of the two when both are
// mapped (system/templates/common/resolveMi.snp:1-28).  Candidates start
// after the previous edge's id (system/templates/funcs/reduceEarlyIdx.snp)
// and stop at the first t > t(e_0) + delta
// (system/templates/common/nextMatchInTask.snp:1-21).
//
// B200 design (not a translation of the reference's per-lane register DFS):
//  * warp-synchronous levels: all 32 lanes of a warp work on the same motif
//    level at once, each on its own partial match, so every load and compare
//    is issued for the whole warp.  A level's matches become child tasks in
//    a per-warp shared-memory buffer (32-byte records with a parent link);
//    whenever 32 are queued the warp descends, processes them as one batch,
//    and returns (depth-first over batches, bounded buffers);
//  * adjacency entries are packed 16-byte records {eid, other, t, pos}: one
//    ld.global.nc.v4 replaces the reference's two dependent gathers
//    (system/templates/common/nextMatchInTask.snp:3-4); per-node ranges are
//    one int4 {out_beg, out_end, in_beg, in_end};
//  * a list opening finds its start in O(1) when the list is the previous
//    edge's own out/in list (the record carries the edge's position in its
//    other list), otherwise by a warp-converged binary search;
//  * when some lanes of a level run dry, idle lanes take interleaved slices
//    of the widest remaining candidate range of that level -- the donor and
//    its thieves each take every parts-th record, so they read neighbouring
//    records in the same step and finish together (one warp shuffle of the
//    donor's state; an exact partition) -- in place of the reference's
//    one-candidate-per-thief split (system/templates/warpBalancing/top.snp)
//    and its host-driven dump/expand rounds (system/templates/tailExpan/Expanding.snp);
//  * the last level reads several records per lane per step (count mode);
//  * a root whose last motif edge has no candidate in its root node's list
//    inside the window is dropped before it takes a lane, the others' windows
//    end at that list's last entry, and the roots that remain are packed into
//    full batches of 32;
//  * same-pair / reverse-pair tails are queued and counted 32 at a time;
//  * enumeration slots are reserved with one warp-aggregated atomicAdd per
//    step (the reference issues one atomicAdd per match,
//    system/tmine/KernelGen.py:505-524).
#include <atomic>

#include "evx_internal.cuh"

namespace evx {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kCap = 64;        // task slots per buffered level per warp
constexpr int kBlock = 128;     // threads per block
constexpr int kWarps = kBlock / 32;
// Records each lane loads per round in a non-last level's scan.
#ifndef EVX_SCAN_WIDE
#define EVX_SCAN_WIDE 2
#endif
constexpr int kScanWide = EVX_SCAN_WIDE;

// Rebalancing hands out interleaved slices (a thief takes every parts-th
// record of the donor's range); 0 hands out contiguous slices instead.
#ifndef EVX_STRIDED
#define EVX_STRIDED 1
#endif

// Check the neighbour signatures before a pair-table lookup.
#ifndef EVX_PAIR_SIG
#define EVX_PAIR_SIG 1
#endif

// A list search for the first record after the previous edge starts from
// the root edge's own position when the list belongs to one of the root
// edge's endpoints (known without a search), galloping up from there; 0:
// a binary search over the whole list.
#ifndef EVX_ROOT_GALLOP
#define EVX_ROOT_GALLOP 1
#endif

// Window end per root from the last motif edge: when that edge has a root
// node as its source (target), it lies in the root node's out-list (in-list)
// after the root edge and inside the window, so every edge of a match is at
// most the last such entry.  When the window holds at most EVX_BOUND_MAX
// of them, that entry's timestamp becomes the root's window end (the same
// matches: the window only loses edges no match can use), and a root with
// none is dropped before it takes a lane.  0: off.
#ifndef EVX_ROOT_BOUND
#define EVX_ROOT_BOUND 1
#endif
#ifndef EVX_BOUND_MAX
#define EVX_BOUND_MAX 32
#endif

// Same-pair / reverse-pair tails inline at a level queue their lookups and
// count them 32 at a time (0: each lane looks its candidates up itself).
#ifndef EVX_TAIL_QUEUE
#define EVX_TAIL_QUEUE 1
#endif

// Roots that pass (not a self-loop, the predicates of a constrained launch,
// the window bound) are packed into full batches of 32 (0: a batch is the
// next 32 roots, passing or not).
#ifndef EVX_ROOT_PACK
#define EVX_ROOT_PACK 1
#endif

// resident blocks per SM the register budget aims for (deeper motifs keep
// more per-level state live)
#ifndef EVX_MINB3
#define EVX_MINB3 10
#endif
#ifndef EVX_MINB4
#define EVX_MINB4 7
#endif
constexpr int min_blocks(int k) { return k <= 3 ? EVX_MINB3 : (k == 4 ? EVX_MINB4 : 4); }

template <int N>
__device__ __forceinline__ int sel(const int (&a)[N], int i) {
  int r = a[0];
#pragma unroll
  for (int q = 1; q < N; q++) r = (i == q) ? a[q] : r;
  return r;
}

template <int N>
__device__ __forceinline__ void put(int (&a)[N], int i, int v) {
#pragma unroll
  for (int q = 0; q < N; q++)
    if (i == q) a[q] = v;
}

__device__ __forceinline__ int ld_eid(const int4 *p) { return __ldg(&p->x); }
__device__ __forceinline__ int ld_t(const int4 *p) { return __ldg(&p->z); }

// First index in [lo, hi) of pair_rec whose timestamp is greater than tl.
__device__ __forceinline__ int pair_first_t_after(const GraphView &g, int lo, int hi, int tl) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&g.pair_rec[mid].y) > tl) hi = mid; else lo = mid + 1;
  }
  return lo;
}

// Count of u->v edges after the previous edge (id > key; t > key in strict
// mode) inside the window, through u's sorted directory of distinct
// out-neighbours.
__device__ __forceinline__ int pair_dir_window(const GraphView &g, int u, int v, int key, int tl,
                                               bool strict);

// Same, galloping up from lo (windows are usually a few entries long).
__device__ __forceinline__ int pair_gallop_t_after(const GraphView &g, int lo, int hi, int tl) {
  int step = 1;
  while (lo < hi) {
    const int probe = min(lo + step - 1, hi - 1);
    if (__ldg(&g.pair_rec[probe].y) > tl) { hi = probe; break; }
    lo = probe + 1;
    step <<= 1;
  }
  return pair_first_t_after(g, lo, hi, tl);
}

// First index in [lo, hi) of pair_rec whose edge id (timestamp in strict
// mode) is greater than key.
__device__ __forceinline__ int pair_first_key_after(const GraphView &g, int lo, int hi, int key,
                                                    bool strict) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const int2 r = __ldg(g.pair_rec + mid);
    if ((strict ? r.y : r.x) > key) hi = mid; else lo = mid + 1;
  }
  return lo;
}

__device__ __forceinline__ int pair_dir_window(const GraphView &g, int u, int v, int key, int tl,
                                               bool strict) {
  int lo = __ldg(g.dir_off + u), hi = __ldg(g.dir_off + u + 1);
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&g.pair_dir[mid].x) < v) lo = mid + 1; else hi = mid;
  }
  const int2 d0 = __ldg(g.pair_dir + lo);
  if (d0.x != v || lo >= __ldg(g.dir_off + u + 1)) return 0;
  const int stop = __ldg(&g.pair_dir[lo + 1].y);
  const int a = pair_first_key_after(g, d0.y, stop, key, strict);
  return pair_gallop_t_after(g, a, stop, tl) - a;
}

// Entries of the run [start, start + len) after the previous edge (edge id >
// key; timestamp > key in strict mode) and inside the window (t <= tl).
__device__ __forceinline__ int pair_window(const GraphView &g, int start, int len, int key, int tl,
                                           bool strict) {
  if (len <= 0) return 0;
  if (len <= 4) {
    int2 r[4];
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (q < len) r[q] = __ldg(g.pair_rec + start + q);
    int c = 0;
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (q < len) c += ((strict ? r[q].y : r[q].x) > key && r[q].y <= tl) ? 1 : 0;
    return c;
  }
  int a = start, b = start + len;
  while (a < b) {
    const int mid = (a + b) >> 1;
    const int2 r = __ldg(g.pair_rec + mid);
    if ((strict ? r.y : r.x) > key) b = mid; else a = mid + 1;
  }
  int c = a, d = start + len;
  while (c < d) {
    const int mid = (c + d) >> 1;
    if (__ldg(&g.pair_rec[mid].y) > tl) d = mid; else c = mid + 1;
  }
  return c - a;
}

// Count a task whose closing edge has few candidates from the closing side.
#ifndef EVX_REVERSE_CLOSE
#define EVX_REVERSE_CLOSE 1
#endif
#ifndef EVX_REV_MAX
#define EVX_REV_MAX 16
#endif
// ... and when the task has more than this many candidates per closing edge
#ifndef EVX_REV_RATIO
#define EVX_REV_RATIO 1
#endif
constexpr int kRevMax = EVX_REV_MAX;  // most closing edges counted that way
constexpr int kRevRatio = EVX_REV_RATIO;

// A new-node last edge's window is counted by range arithmetic when more than
// this many records per already-mapped node remain (one pair probe each).
#ifndef EVX_ARITH_RECS
#define EVX_ARITH_RECS 8
#endif
constexpr int kArithRecs = EVX_ARITH_RECS;

// First position in [lo, hi) of an adjacency list whose timestamp is
// greater than tl, galloping up from lo (windows are usually short).
__device__ __forceinline__ int list_first_t_after(const int4 *lst, int lo, int hi, int tl) {
  int step = 1;
  while (lo < hi) {
    const int probe = min(lo + step - 1, hi - 1);
    if (ld_t(lst + probe) > tl) { hi = probe; break; }
    lo = probe + 1;
    step <<= 1;
  }
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ld_t(lst + mid) > tl) hi = mid; else lo = mid + 1;
  }
  return lo;
}

// First position in [lo, hi) of an adjacency list whose edge id is greater
// than key, galloping up from lo.
__device__ __forceinline__ int list_first_eid_after(const int4 *lst, int lo, int hi, int key) {
  int step = 1;
  while (lo < hi) {
    const int probe = min(lo + step - 1, hi - 1);
    if (ld_eid(lst + probe) > key) { hi = probe; break; }
    lo = probe + 1;
    step <<= 1;
  }
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ld_eid(lst + mid) > key) hi = mid; else lo = mid + 1;
  }
  return lo;
}

// Entries of the pair run [start, start + len) whose edge id lies in [klo, khi].
__device__ __forceinline__ int pair_count_eids(const GraphView &g, int start, int len, int klo, int khi) {
  if (len <= 0) return 0;
  int a = start, b = start + len;
  while (a < b) {
    const int mid = (a + b) >> 1;
    if (__ldg(&g.pair_rec[mid].x) >= klo) b = mid; else a = mid + 1;
  }
  int c = a, d = start + len;
  while (c < d) {
    const int mid = (c + d) >> 1;
    if (__ldg(&g.pair_rec[mid].x) > khi) d = mid; else c = mid + 1;
  }
  return c - a;
}

// Per-warp shared state.
//   root[r]           = {u, v, tl, e0} of the batch's root on lane r
//   task[l-1][s][0/1] = {parent, src, dst, eid}, {t, pos in out_rec, pos in in_rec, root}
//                       of a partial match waiting at level l (l = 1 .. k-2)
//   save[l][lane]     = scan state of level l parked while the warp descends
template <int K>
struct alignas(16) WarpSmem {
  QueryDesc q;             // the warp's current query
  int4 root[32];
  int4 task[(K > 2) ? (K - 2) : 1][kCap][2];
  int4 save[(K > 2) ? (K - 2) : 1][32][2];
  int nb[K];
  int cur_q;               // index of the current query in the launch
  int halt;                // set when the current query stops early (limit or cap)
};

// The previous matched edge of a task (what the next list opening needs).
struct Prev {
  int eid, t, src, dst, pop, pip;
};

template <int K, bool ENUM, bool EXACT, bool PS, bool CS>
struct Searcher {
  static constexpr int L = K - 1;          // levels; level l opens motif edge l + 1
  static constexpr int N = K + 1;          // motif nodes <= k + 1
  static constexpr int KE = ENUM ? K : 1;
  static constexpr int WIDE = ENUM ? 1 : 4;  // records per lane per last-level step

  const GraphView &g;
  const MotifPlan &plan;   // the current query's plan (per-warp copy in shared memory)
  const EnumArgs &ea;
  const LaunchArgs &la;
  WarpSmem<K> &sm;
  const int lane;
  const unsigned lt;
  // the current query's options (reloaded when the warp switches queries)
  // the current query's options: kQ* flags and rebalance interval in
  // registers, the rest read from its shared-memory copy
  int qf = 0;
  int si = 0;
  // motif edges of the current query: K itself when the launch has one
  // motif size (EXACT), else the table entry's
  __device__ __forceinline__ int kr() const { return EXACT ? K : sm.q.plan.k; }
  __device__ __forceinline__ bool strict_() const { return (qf & kQStrict) != 0; }
  unsigned long long cnt;
  unsigned cand;  // adjacency records examined inside the window since the last meter update

  __device__ Searcher(const GraphView &g_, const MotifPlan &p_, const EnumArgs &e_, const LaunchArgs &la_,
                      WarpSmem<K> &s_, int lane_)
      : g(g_), plan(p_), ea(e_), la(la_), sm(s_), lane(lane_), lt((1u << lane_) - 1u), cnt(0), cand(0) {}

  // Add this warp's examined records to the current query's meter; returns
  // the meter after the add.
  __device__ __forceinline__ unsigned long long meter_add() {
    unsigned long long c = cand;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(kFull, c, o);
    unsigned long long tot = 0;
    if (lane == 0) tot = atomicAdd(la.meter + sm.cur_q, c) + c;
    cand = 0;
    return __shfl_sync(kFull, tot, 0);
  }

  // Whether the current query has stopped: its enumeration cap was reached,
  // or (with a work limit) its meter passed the limit.  The meter counts the
  // adjacency records the search examines inside their time windows (not
  // the one record past a window that ends each scan, nor binary-search
  // probes): every such record is examined exactly once however the scans
  // are split between lanes, so the meter's final value is fixed by the
  // graph and the query.  Lanes add to it once one holds 64 records (so
  // the records not yet added stay below 64 x the lanes of the grid); the
  // total returned by that add is what is compared, so a query is stopped
  // only once its final meter is known to exceed the limit.
  __device__ __forceinline__ bool halted() {
    if (sm.halt) return true;
    if constexpr (ENUM) {
      if (!ea.exact_total && *(volatile int *)ea.stop != 0) return true;
    }
    if (!la.limit) return false;
    if (!__any_sync(kFull, cand >= 64u)) return false;
    return meter_add() > la.limit;
  }

  __device__ __forceinline__ void set_query(const QueryDesc &q) {
    qf = q.flags;
    si = q.steal_interval;
  }

  // Node images and edge ids of the partial match in slot s of level l.
  template <int l>
  __device__ __forceinline__ void reconstruct(int s, int (&m)[N], int (&e)[KE], Prev &p, int &root) {
#pragma unroll
    for (int q = 0; q < N; q++) m[q] = -1;
    if constexpr (l == 0) {
      root = s;
    } else {
      const int4 a0 = sm.task[l - 1][s][0], a1 = sm.task[l - 1][s][1];
      p.eid = a0.w; p.t = a1.x; p.src = a0.y; p.dst = a0.z; p.pop = a1.y; p.pip = a1.z;
      root = a1.w;
      int cur = s;
#pragma unroll
      for (int j = l; j >= 1; j--) {
        const int4 t0 = sm.task[j - 1][cur][0];
        const int w = plan.info[j - 1];  // level j-1 matched motif edge j
        const int kind = plan_kind(w);
        if (kind == 0) put(m, plan_nm(w), t0.y);
        else if (kind == 1) put(m, plan_nm(w), t0.z);
        if (ENUM) put(e, j, t0.w);
        cur = t0.x;
      }
    }
    const int4 r = sm.root[root];
    m[0] = r.x;
    m[1] = r.y;
    if (ENUM) e[0] = r.w;
    if constexpr (l == 0) {
      (void)p;
    }
  }

  // First position of out(x) / in(x) after the previous edge p when it is
  // known without a search (p is in the list, or p's other endpoint is x),
  // else -1.
  __device__ __forceinline__ int out_start(const Prev &p, int x) const {
    return p.src == x ? p.pop + 1 : (p.dst == x ? __ldg(g.cross_out + p.eid) : -1);
  }
  __device__ __forceinline__ int in_start(const Prev &p, int x) const {
    return p.dst == x ? p.pip + 1 : (p.src == x ? __ldg(g.cross_in + p.eid) : -1);
  }

  // First position of out(x) / in(x) after the root edge (x one of its
  // endpoints), else -1: every later edge of the partial match comes after
  // it, so a search for the first record after the previous edge can start
  // there.
  __device__ __forceinline__ int after_root(int root, int x, bool outl) const {
    const int4 rt = sm.root[root];
    if (outl) return x == rt.x ? __ldg(&g.edges[rt.w].w) + 1 : (x == rt.y ? __ldg(g.cross_out + rt.w) : -1);
    return x == rt.y ? __ldg(g.inpos + rt.w) + 1 : (x == rt.x ? __ldg(g.cross_in + rt.w) : -1);
  }

  // Constrained queries (CS): a candidate also needs its edge predicate and,
  // when it maps a new motif node (want < 0), that node's predicate (bit nmc
  // of its mask: the new node's index is the number mapped before it).
  __device__ __forceinline__ bool cons_ok(int eid, int node, int want, int nmc) const {
    if constexpr (!CS) {
      return true;
    } else {
      if (la.cons.edge_ok && !__ldg(la.cons.edge_ok + eid)) return false;
      if (want < 0 && la.cons.node_ok && !((__ldg(la.cons.node_ok + node) >> nmc) & 1)) return false;
      return true;
    }
  }

  __device__ __forceinline__ bool structural_ok(int node, int want, int nmc, const int (&m)[N]) const {
    if (want >= 0) return node == want;
    bool ok = true;
#pragma unroll
    for (int q = 0; q < N; q++) ok = ok && !(q < nmc && m[q] == node);
    return ok;
  }

  // Push one child partial match (found at level l) into level l+1's buffer.
  template <int l>
  __device__ __forceinline__ void push_children(bool push, int parent, const int4 &rc, bool out, int base,
                                                int pos_found, int root) {
    const unsigned pm = __ballot_sync(kFull, push);
    if (!pm) return;
    const int nb = sm.nb[l + 1];
    if (push) {
      const int s = nb + __popc(pm & lt);
      const int src = out ? base : rc.y, dst = out ? rc.y : base;
      const int pw = rc.w & kPosMask;
      const int pop = out ? pos_found : pw, pip = out ? pw : pos_found;
      sm.task[l][s][0] = make_int4(parent, src, dst, rc.x);
      sm.task[l][s][1] = make_int4(rc.z, pop, pip, root);
    }
    __syncwarp();
    if (lane == 0) sm.nb[l + 1] = nb + __popc(pm);
    __syncwarp();
  }

  // Process one queued batch (up to 32 tasks) of level l+1, then move the
  // tasks that were not in the batch to the front of the buffer.
  template <int l>
  __device__ __forceinline__ void descend() {
    if constexpr (l + 1 < L) {
      if (halted()) {
        // drop the queued tasks; the caller ends its scan on sm.halt
        __syncwarp();
        if (lane == 0) { sm.halt = 1; sm.nb[l + 1] = 0; }
        __syncwarp();
        return;
      }
      const int nb = sm.nb[l + 1];
      const int take = nb < 32 ? nb : 32;
      level<l + 1>(lane < take, lane, take);
      __syncwarp();
      const int rest = sm.nb[l + 1] - take;  // rest < 32: one record per lane at most
      int4 a0 = make_int4(0, 0, 0, 0), a1 = a0;
      if (lane < rest) { a0 = sm.task[l][take + lane][0]; a1 = sm.task[l][take + lane][1]; }
      __syncwarp();
      if (lane < rest) { sm.task[l][lane][0] = a0; sm.task[l][lane][1] = a1; }
      if (lane == 0) sm.nb[l + 1] = rest;
      __syncwarp();
    }
  }

  // One batch at level l: lanes with 'has' own the partial match in slot
  // 'slot' (root lane for l = 0).  nbatch is informational.
  template <int l>
  __device__ __forceinline__ void level(bool has, int slot, int nbatch) {
    (void)nbatch;
    int m[N];
    int e[KE];
#pragma unroll
    for (int q = 0; q < KE; q++) e[q] = 0;
    Prev p = {0, 0, 0, 0, 0, 0};
    int root = lane;
    if (has) reconstruct<l>(slot, m, e, p, root);
    else {
#pragma unroll
      for (int q = 0; q < N; q++) m[q] = -1;
    }
    if constexpr (l == 0) {
      if (has) {
        const int4 r = sm.root[slot];
        const int e0 = r.w;
        const int4 ed = __ldg(g.edges + e0);
        p.eid = e0; p.t = ed.z; p.src = ed.x; p.dst = ed.y; p.pop = ed.w; p.pip = __ldg(g.inpos + e0);
      }
    }
    int tl = sm.root[root].z;
    if constexpr (CS) {
      // temporal gaps: motif edge l + 1 ends its window gap[l] after the
      // previous edge (edge 1: after the root, even past delta; later ones
      // never past t(e_0) + delta)
      if (la.cons.has_gap && has) tl = l == 0 ? p.t + la.cons.gap[0] : min(p.t + la.cons.gap[l], tl);
    }

    // ---------------------------- last level through the pair hash table ----
    if (!ENUM && (qf & kQPairHash) && l == kr() - 2) {
      // the closing last edge of each lane's task: one hash probe sequence
      // for its pair's run, then the run's entries after the previous edge
      // and inside the window (runs are short; 32 lanes probe in parallel)
      if (has) {
        const int w = plan.info[l];
        const int ia = sel(m, plan_a(w)), ib = sel(m, plan_b(w));
        if (EVX_PAIR_SIG == 0 || pair_maybe(g, ia, ib)) {
          const int2 f = pair_find(g, ia, ib);
          cnt += (unsigned long long)pair_window(g, f.x, f.y, strict_() ? p.t : p.eid, tl, strict_());
        }
        ++cand;  // one lookup per task
      }
      return;
    }

    // --------------------------- last level through the pair directory ----
    if (!ENUM && (qf & kQPairDir) && l == kr() - 2) {
      // the closing last edge of each lane's task: count its static pair's
      // run inside the window (converged across the batch's 32 tasks)
      if (has) {
        const int w = plan.info[l];
        const int ia = sel(m, plan_a(w)), ib = sel(m, plan_b(w));
        const int tlc = sm.root[root].z;
        cnt += (unsigned long long)pair_dir_window(g, ia, ib, strict_() ? p.t : p.eid, tlc, strict_());
        ++cand;  // one directory lookup per task
      }
      return;
    }

    // ------------------------------------------------------- open list ----
    const int w = plan.info[l];
    const int kind = plan_kind(w);
    const int nmc = plan_nm(w);
    int pos = 0, end = 0, want = -1, base = 0;
    int stride = 1;  // distance between this lane's records (interleaved slices)
    bool out = true;
    bool prun = false;  // the range is a run of pair_rec (the edge's static pair), not a list
    int blo = 0, bhi = 0, gstep = 0;
    bool searching = false;
    if (PS && has && kind == 2 && (qf & kQPairScan)) {
      // both endpoints are mapped: walk the run of the static edge (ia, ib)
      // after the previous edge; every entry matches structurally.  The run
      // is located from the previous edge itself when it is that pair or its
      // reverse, else by one hash probe (after the signature filter).
      const int ia = sel(m, plan_a(w)), ib = sel(m, plan_b(w));
      prun = true; out = true; base = ia; want = ib;
      int lo, hi;
      if (ia == p.src && ib == p.dst) {
        const int2 pl = __ldg(g.pair_loc + p.eid);
        lo = pl.x + 1; hi = pl.y;
        if (strict_()) lo = pair_first_t_after(g, lo, hi, p.t);
      } else if (ia == p.dst && ib == p.src) {
        const int2 rl = __ldg(g.rev_loc + p.eid);
        lo = rl.x; hi = rl.y;
        if (strict_()) lo = pair_first_t_after(g, lo, hi, p.t);
      } else {
        const int2 f = (EVX_PAIR_SIG == 0 || pair_maybe(g, ia, ib)) ? pair_find(g, ia, ib) : make_int2(0, 0);
        hi = f.x + f.y;
        lo = pair_first_key_after(g, f.x, hi, strict_() ? p.t : p.eid, strict_());
      }
      pos = lo; end = hi;
    } else if (has) {
      const int ia = sel(m, plan_a(w)), ib = sel(m, plan_b(w));
      int lo, hi, sc;
      if (kind == 2) {
        const int4 ri = __ldg(g.node_rng + ib);
        const int4 ro = __ldg(g.node_rng + ia);
        if (ri.w - ri.z < ro.y - ro.x) {
          out = false; base = ib; want = ia; lo = ri.z; hi = ri.w;
          sc = in_start(p, ib);
        } else {
          out = true; base = ia; want = ib; lo = ro.x; hi = ro.y;
          sc = out_start(p, ia);
        }
      } else if (kind == 1) {
        const int4 r = __ldg(g.node_rng + ia);
        out = true; base = ia; lo = r.x; hi = r.y;
        sc = out_start(p, ia);
      } else {
        const int4 r = __ldg(g.node_rng + ib);
        out = false; base = ib; lo = r.z; hi = r.w;
        sc = in_start(p, ib);
      }
      end = hi;
      if (!strict_() && sc >= 0) {
        pos = sc;
      } else if (lo < hi) {
        blo = lo; bhi = hi; searching = true;
        if (EVX_ROOT_GALLOP && l > 0 && !strict_()) {
          const int fr = after_root(root, base, out);
          if (fr >= 0) { blo = fr; gstep = 1; }
          if (blo >= bhi) { searching = false; pos = bhi; }
        }
      } else {
        pos = hi;
      }
    }
    // first record after the previous edge (by id; by time in strict mode):
    // galloping up from the root edge's position while gstep > 0, then
    // halving
    {
      const int key = strict_() ? p.t : p.eid;
      while (__any_sync(kFull, searching)) {
        if (searching) {
          const int4 *lst = out ? g.out_rec : g.in_rec;
          const int mid = gstep > 0 ? min(blo + gstep - 1, bhi - 1) : (blo + bhi) >> 1;
          const int v = strict_() ? ld_t(lst + mid) : ld_eid(lst + mid);
          if (v > key) { bhi = mid; gstep = 0; } else { blo = mid + 1; gstep <<= 1; }
          if (blo >= bhi) { searching = false; pos = blo; }
        }
      }
    }

    int steps = 0;
    if (l == kr() - 2 || l == L - 1) {
      // ------------------------------------------------ last level ----
      bool arith = true;  // the range-arithmetic check is still to be made
      int chk = 0;
      while (true) {
        const unsigned act = __ballot_sync(kFull, pos < end);
        if (!act) break;
        if (la.limit && ((++chk) & 63) == 0 && halted()) {
          // a long scan with a work limit: the query passed it; stop here
          pos = end;
          __syncwarp();
          if (lane == 0) sm.halt = 1;
          __syncwarp();
          break;
        }
        if (act != kFull && si && ((++steps) & (si - 1)) == 0)
          rebalance(act, pos, end, stride, want, out, prun, base, slot, root, tl, m, e);
        bool emit = false;
        int last_eid = 0;
        const int st = EVX_STRIDED ? stride : 1;
        if (pos < end) {
          const int4 *lst = out ? g.out_rec : g.in_rec;
          int4 rr[WIDE];
#pragma unroll
          for (int q = 0; q < WIDE; q++) {
            if (q == 0 || pos + q * st < end) {
              if (prun) {
                const int2 pr = __ldg(g.pair_rec + pos + q * st);
                rr[q] = make_int4(pr.x, want, pr.y, 0);
              } else {
                rr[q] = __ldg(lst + pos + q * st);
              }
            }
          }
#pragma unroll
          for (int q = 0; q < WIDE; q++) {
            if (pos < end) {
              pos += st;
              if (rr[q].z > tl) {
                pos = end;
              } else {
                ++cand;
                if (structural_ok(rr[q].y, want, nmc, m) && cons_ok(rr[q].x, rr[q].y, want, nmc)) {
                  ++cnt;
                  if (ENUM) { emit = true; last_eid = rr[q].x; }
                }
              }
            }
          }
          if constexpr (!ENUM) {
            if (want < 0 && pos < end && arith && (qf & kQNewArith) && st == 1) {
              // a last edge that maps a new node, and the window goes on past
              // this step: when the rest of the window is long, it counts
              // every record except those whose other endpoint is already
              // mapped, i.e. the entries of the pairs (base, m_j) (or
              // (m_j, base)) inside the same edge-id range; a short rest is
              // scanned (each pair costs a table probe)
              arith = false;
              const int wend = list_first_t_after(lst, pos, end, tl);
              if (wend - pos <= kArithRecs * nmc) {
                end = wend;
              } else {
                const int klo = ld_eid(lst + pos), khi = ld_eid(lst + wend - 1);
                int sub = 0;
#pragma unroll
                for (int j = 0; j < N; j++) {
                  if (j < nmc) {
                    const int a_ = out ? base : m[j], b_ = out ? m[j] : base;
                    if (pair_maybe(g, a_, b_)) {
                      const int2 f = pair_find(g, a_, b_);
                      sub += pair_count_eids(g, f.x, f.y, klo, khi);
                    }
                  }
                }
                cnt += (unsigned long long)(wend - pos - sub);
                cand += (unsigned)(wend - pos);  // the meter covers counted records too
                pos = end;
              }
            }
          }
        }
        if constexpr (ENUM) {
          if (emit_row(emit, e, last_eid)) {
            // the cap is reached: end this scan and unwind the levels above
            pos = end;
            __syncwarp();
            if (lane == 0) sm.halt = 1;
            __syncwarp();
            break;
          }
        }
      }
    } else if constexpr (l < L - 1) {
      // --------------------------------- scan, queue children, descend ----
      // The level before the last one counts a closing last edge inline by
      // range arithmetic on the pair index (count mode only).
      const bool inline_here = (l == kr() - 3) && !ENUM && (qf & (kQInlineLast | kQSamePair | kQRevPair));
      const int wl = plan.info[kr() - 2];
      const int la = plan_a(wl), lb = plan_b(wl);
      int ca = -1, cb = -1, ctl = 0, cs = 0, cub = 0, ckey = 0;  // this lane's pair cursor
      if (inline_here && (qf & kQInlineLast) && has && pos < end) {
        // the closing pair is fixed for the task: place the cursor on its
        // run's entries after the previous edge inside the window once; when
        // there are none, no candidate of the task can close and its scan is
        // skipped
        // (the previous edge's own pair, or its reverse, is located per edge
        // without a table lookup)
        const int ia = sel(m, la), ib = sel(m, lb);
        const int key = strict_() ? p.t : p.eid;
        int lo, hi;
        if (ia == p.src && ib == p.dst) {
          const int2 pl = __ldg(g.pair_loc + p.eid);
          lo = pl.x + 1; hi = pl.y;
          if (strict_()) lo = pair_first_t_after(g, lo, hi, p.t);
        } else if (ia == p.dst && ib == p.src) {
          const int2 rl = __ldg(g.rev_loc + p.eid);
          lo = rl.x; hi = rl.y;
          if (strict_()) lo = pair_first_t_after(g, lo, hi, p.t);
        } else {
          const int2 f = (EVX_PAIR_SIG == 0 || pair_maybe(g, ia, ib)) ? pair_find(g, ia, ib) : make_int2(0, 0);
          lo = pair_first_key_after(g, f.x, f.x + f.y, key, strict_());
          hi = f.x + f.y;
        }
        ca = ia; cb = ib; ctl = tl; ckey = key;
        cs = lo;
        cub = pair_gallop_t_after(g, lo, hi, tl);
        if (cs >= cub) pos = end;
      }
      if (l == kr() - 3 && plan_kind(wl) == 2 && (la < nmc) != (lb < nmc) &&
          !(qf & (kQInlineLast | kQNoPrune)) && has && pos < end && !prun) {
        // the closing edge has one endpoint mapped before this level, fixed
        // for the task: when that node's list (out-list of a source, in-list
        // of a destination) has no entry after the previous edge inside the
        // window, no candidate of the task can close, so its scan is skipped
        const bool fa = la < nmc;
        const int x = sel(m, fa ? la : lb);
        const int4 r = __ldg(g.node_rng + x);
        int lo = fa ? r.x : r.z, hi = fa ? r.y : r.w;
        const int4 *lst = fa ? g.out_rec : g.in_rec;
        const int key = strict_() ? p.t : p.eid;
        const int known = strict_() ? -1 : (fa ? out_start(p, x) : in_start(p, x));
        const int fr = (EVX_ROOT_GALLOP && known < 0 && !strict_() && l > 0) ? after_root(root, x, fa) : -1;
        if (known >= 0) lo = known;
        else if (fr >= 0) lo = list_first_eid_after(lst, fr, hi, key);
        else {
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const int v = strict_() ? ld_t(lst + mid) : ld_eid(lst + mid);
            if (v > key) hi = mid; else lo = mid + 1;
          }
          hi = fa ? r.y : r.w;
        }
        if (lo >= hi || ld_t(lst + lo) > tl) {
          pos = end;
        } else if (EVX_REVERSE_CLOSE && !ENUM && !CS && !strict_() && !(qf & (kQSamePair | kQRevPair))) {
          // Few closing edges: count the task from the closing side.  Each
          // closing edge e2 (x, c) inside the window pairs with the
          // candidates e1 of this level that map the same new node c and
          // come between the previous edge and e2, i.e. the entries of the
          // pair (base, c) (or (c, base)) with edge id in (p, e2).  Taken
          // when the window holds at most kRevMax closing edges and more than
          // kRevRatio candidates per closing edge.
          // (the window's closing edges are counted by a gallop bounded at
          // kRevMax + 1 records; each closing record is loaded when used)
          const int cap_hi = min(hi, lo + kRevMax + 1);
          const int n2 = list_first_t_after(lst, lo, cap_hi, tl) - lo;
          const bool more = n2 > kRevMax;
          const int4 *lst1 = out ? g.out_rec : g.in_rec;
          if (!more && pos + kRevRatio * n2 < end && ld_t(lst1 + pos + kRevRatio * n2) <= tl) {
            for (int j = 0; j < n2; j++) {
              const int4 c3 = __ldg(lst + lo + j);
              const int cn = c3.y;
              bool fresh = true;
#pragma unroll
              for (int q = 0; q < N; q++) fresh = fresh && !(q < nmc && m[q] == cn);
              const int a_ = out ? base : cn, b_ = out ? cn : base;
              if (fresh && pair_maybe(g, a_, b_)) {
                const int2 f = pair_find(g, a_, b_);
                cnt += (unsigned long long)pair_count_eids(g, f.x, f.y, p.eid + 1, c3.x - 1);
              }
            }
            cand += (unsigned)(n2 + 1);
            pos = end;
          }
        }
      }
      int chk = 0;
      while (true) {
        const unsigned act = __ballot_sync(kFull, pos < end);
        if (!inline_here) {
          const int nb = sm.nb[l + 1];
          if (nb >= 32 || (!act && nb > 0)) {
            // park this level's state in shared memory while the warp descends,
            // so none of it stays live in registers across the nested batch
            sm.save[l][lane][0] = make_int4(pos, end, want, base);
            // flags word: steps (mod 256, only its low bits matter) | stride (< 2^20) | prun | out
            sm.save[l][lane][1] = make_int4(slot, root, tl, (int)(((unsigned)steps & 0xffu) << 24) |
                                                                ((EVX_STRIDED ? stride : 1) << 2) | (prun ? 2 : 0) |
                                                                (out ? 1 : 0));
            __syncwarp();
            descend<l>();
            const int4 s0 = sm.save[l][lane][0], s1 = sm.save[l][lane][1];
            pos = s0.x; end = s0.y; want = s0.z; base = s0.w;
            slot = s1.x; root = s1.y; tl = s1.z; out = (s1.w & 1) != 0; prun = PS && (s1.w & 2) != 0;
            steps = (int)((unsigned)s1.w >> 24);
            stride = EVX_STRIDED ? (s1.w >> 2) & 0x3fffff : 1;
            if (sm.halt) pos = end;  // the query stopped: unwind this level too
            Prev dummy;
            int rr;
            if (pos < end) reconstruct<l>(slot, m, e, dummy, rr);
            continue;
          }
        }
        if (!act) break;
        if (this->la.limit && ((++chk) & 63) == 0 && halted()) {  // (la here: the last edge's a)
          // a long scan with a work limit: the query passed it; drop its
          // queued tasks and unwind (its result is discarded)
          pos = end;
          __syncwarp();
          if (lane == 0) { sm.halt = 1; sm.nb[l + 1] = 0; }
          __syncwarp();
          break;
        }
        if (act != kFull && si && ((++steps) & (si - 1)) == 0)
          rebalance(act, pos, end, stride, want, out, prun, base, slot, root, tl, m, e);
        const int st = EVX_STRIDED ? stride : 1;
        // the next kScanWide records of every lane's range in one round of
        // loads (one memory latency instead of kScanWide), then processed
        // one at a time; records not processed before a descend are
        // loaded again after it.  A pair run's entries {eid, t} become
        // out-list records of its source: {eid, target, t, position in
        // in_rec}, with the position in out_rec beside them (pf).
        int4 rw[kScanWide];
        int pf[kScanWide];
        {
          const int4 *lst = out ? g.out_rec : g.in_rec;
#pragma unroll
          for (int q = 0; q < kScanWide; q++) {
            rw[q] = make_int4(0, 0, 0, 0);
            pf[q] = pos + q * st;
            if (pos + q * st < end) {
              if (prun) {
                const int2 pr = __ldg(g.pair_rec + pos + q * st);
                rw[q] = make_int4(pr.x, want, pr.y, 0);
              } else {
                rw[q] = __ldg(lst + pos + q * st);
              }
            }
          }
          if (prun && !inline_here) {
#pragma unroll
            for (int q = 0; q < kScanWide; q++) {
              if (pos + q * st < end && rw[q].z <= tl) {
                rw[q].w = __ldg(g.inpos + rw[q].x);
                pf[q] = __ldg(&g.edges[rw[q].x].w);  // edges[] positions carry no flags
              }
            }
          }
        }
        if (inline_here) {
          // count only, nothing queued: take every loaded record's verdict
          // first, then issue the closing-edge lookups of all of them
          bool ok[kScanWide];
#pragma unroll
          for (int q = 0; q < kScanWide; q++) {
            ok[q] = false;
            if (pos < end) {
              pos += st;
              if (rw[q].z > tl) {
                pos = end;
              } else {
                ++cand;
                ok[q] = structural_ok(rw[q].y, want, nmc, m) && cons_ok(rw[q].x, rw[q].y, want, nmc);
              }
            }
          }
          if (qf & (kQSamePair | kQRevPair)) {
            // the last edge repeats the matched edge's endpoints (or reverses
            // them): count the entries of that edge's own pair run (or of the
            // reverse pair's run) after the edge and inside the window
            const bool rev = (qf & kQRevPair) != 0;
            // a candidate whose record says its own pair's run (top bit) or
            // its reverse pair's run (kRevLater) has no entry after it adds
            // nothing: skip its lookup
            const int later = rev ? kRevLater : (int)0x80000000u;
            if (EVX_TAIL_QUEUE && !strict_()) {
              // queue them (edge id, window end) in the next level's unused
              // task buffer and count them 32 at a time
#pragma unroll
              for (int q = 0; q < kScanWide; q++) {
                const bool push = ok[q] && (prun || (rw[q].w & later));
                const unsigned pm = __ballot_sync(kFull, push);
                if (pm) {
                  const int nb = sm.nb[l + 1];
                  if (push) sm.task[l][nb + __popc(pm & lt)][0] = make_int4(rw[q].x, tl, 0, 0);
                  __syncwarp();
                  if (lane == 0) sm.nb[l + 1] = nb + __popc(pm);
                  __syncwarp();
                  if (nb + __popc(pm) >= 32) tail_batch<l>(rev, false);
                }
              }
            } else {
              int2 pl[kScanWide];
#pragma unroll
              for (int q = 0; q < kScanWide; q++) {
                if (!prun && !(rw[q].w & later)) ok[q] = false;
                pl[q] = ok[q] ? __ldg((rev ? g.rev_loc : g.pair_loc) + rw[q].x) : make_int2(0, 0);
              }
#pragma unroll
              for (int q = 0; q < kScanWide; q++) {
                if (ok[q]) {
                  int lo = rev ? pl[q].x : pl[q].x + 1;
                  if (strict_()) lo = pair_first_t_after(g, lo, pl[q].y, rw[q].z);
                  cnt += (unsigned long long)(pair_gallop_t_after(g, lo, pl[q].y, tl) - lo);
                }
              }
            }
          } else {
            // the last edge joins two nodes mapped before this level, so its
            // pair run is fixed for the task: a cursor into it only moves
            // forward as this lane's candidates advance
#pragma unroll
            for (int q = 0; q < kScanWide; q++) {
              if (ok[q]) {
                const int ia = sel(m, la), ib = sel(m, lb);
                const int key = strict_() ? rw[q].z : rw[q].x;
                if (ia != ca || ib != cb || tl != ctl || key < ckey) {
                  const int2 f = pair_find(g, ia, ib);
                  ca = ia; cb = ib; ctl = tl;
                  cub = pair_first_t_after(g, f.x, f.x + f.y, tl);
                  cs = pair_first_key_after(g, f.x, cub, key, strict_());
                } else {
                  // a few steps forward; fall back to a search for long jumps
                  int steps_left = 4;
                  while (cs < cub && steps_left-- > 0 &&
                         (strict_() ? __ldg(&g.pair_rec[cs].y) : __ldg(&g.pair_rec[cs].x)) <= key) ++cs;
                  if (steps_left < 0) cs = pair_first_key_after(g, cs, cub, key, strict_());
                }
                ckey = key;
                cnt += (unsigned long long)(cub - cs);
              }
            }
          }
        } else {
#pragma unroll
          for (int q = 0; q < kScanWide; q++) {
            bool push = false;
            const int4 rc = rw[q];
            if (pos < end) {
              pos += st;
              if (rc.z > tl) {
                pos = end;
              } else {
                ++cand;
                push = structural_ok(rc.y, want, nmc, m) && cons_ok(rc.x, rc.y, want, nmc);
              }
            }
            push_children<l>(push, slot, rc, out, base, pf[q], root);
            if (sm.nb[l + 1] >= 32) break;  // descend before the next push
          }
        }
      }
      if (EVX_TAIL_QUEUE && inline_here && (qf & (kQSamePair | kQRevPair)) && !strict_()) {
        // the queued tail lookups left over (none when the query stopped)
        if (sm.halt) {
          __syncwarp();
          if (lane == 0) sm.nb[l + 1] = 0;
          __syncwarp();
        } else {
          tail_batch<l>((qf & kQRevPair) != 0, true);
        }
      }
    }
  }

  // Count the queued same-pair / reverse-pair tail lookups of level l (in
  // the task buffer of level l + 1, which an inline level leaves unused):
  // 32 at a time, each lane one entry {edge id, window end}: the entries of
  // the edge's own pair run (reverse pair's run) after it and inside the
  // window.  all: until the queue is empty, else one batch.  At most 63
  // entries are queued when it is called.
  template <int l>
  __device__ __forceinline__ void tail_batch(bool rev, bool all) {
    if constexpr (l < L - 1) {
      while (true) {
        const int nb = sm.nb[l + 1];
        if (nb == 0) break;
        const int take = nb < 32 ? nb : 32;
        if (lane < take) {
          const int4 qe = sm.task[l][lane][0];
          const int2 pl = __ldg((rev ? g.rev_loc : g.pair_loc) + qe.x);
          const int lo = rev ? pl.x : pl.x + 1;
          cnt += (unsigned long long)(pair_gallop_t_after(g, lo, pl.y, qe.y) - lo);
        }
        __syncwarp();
        const int rest = nb - take;
        int4 a = make_int4(0, 0, 0, 0);
        if (lane < rest) a = sm.task[l][take + lane][0];
        __syncwarp();
        if (lane < rest) sm.task[l][lane][0] = a;
        if (lane == 0) sm.nb[l + 1] = rest;
        __syncwarp();
        if (!all) break;
      }
    }
  }

  // Idle lanes take equal slices of the widest remaining range at this level
  // (contiguous, or interleaved with EVX_STRIDED: every parts-th record).
  template <int NN, int EE>
  __device__ __forceinline__ void rebalance(unsigned act, int &pos, int &end, int &stride, int &want, bool &out,
                                            bool &prun, int &base, int &slot, int &root, int &tl,
                                            int (&m)[NN], int (&e)[EE]) {
    const int st = EVX_STRIDED ? stride : 1;
    const int width = EVX_STRIDED ? (end - pos + st - 1) / st : end - pos;
    const unsigned wmax = __reduce_max_sync(kFull, (unsigned)(width > 0 ? width : 0));
    if ((int)wmax < sm.q.min_split) return;
    const int donor = __ffs(__ballot_sync(kFull, (unsigned)width == wmax)) - 1;
    const unsigned idle = ~act;
    const int nthief = min(__popc(idle), (int)wmax - 1);
    if (nthief <= 0) return;
    const int parts = nthief + 1;
    const int rank = __popc(idle & lt);
    const bool thief = ((idle >> lane) & 1u) && rank < nthief;
    const int d_st = EVX_STRIDED ? __shfl_sync(kFull, st, donor) : 1;
    if (EVX_STRIDED && (long long)d_st * parts >= (1 << 20)) return;  // a stride must fit its 20 bits
    const int p0 = __shfl_sync(kFull, pos, donor);
#pragma unroll
    for (int q = 0; q < NN; q++) {
      const int x = __shfl_sync(kFull, m[q], donor);
      if (thief) m[q] = x;
    }
    if (ENUM) {
#pragma unroll
      for (int q = 0; q < EE; q++) {
        const int x = __shfl_sync(kFull, e[q], donor);
        if (thief) e[q] = x;
      }
    }
    const int d_want = __shfl_sync(kFull, want, donor);
    const int d_out = __shfl_sync(kFull, (int)out | ((PS && prun) ? 2 : 0), donor);
    const int d_base = __shfl_sync(kFull, base, donor);
    const int d_slot = __shfl_sync(kFull, slot, donor);
    const int d_root = __shfl_sync(kFull, root, donor);
    const int d_tl = __shfl_sync(kFull, tl, donor);
    const int w = (int)wmax;
    if (EVX_STRIDED) {
      // interleaved: record i of the donor's remaining range goes to part
      // i mod parts; all parts keep the donor's end
      const int d_end = __shfl_sync(kFull, end, donor);
      if (thief) {
        want = d_want; out = (d_out & 1) != 0; prun = PS && (d_out & 2) != 0; base = d_base; slot = d_slot;
        root = d_root; tl = d_tl;
        pos = p0 + (rank + 1) * d_st;
        end = d_end;
        stride = d_st * parts;
      }
      if (lane == donor) stride = d_st * parts;
      return;
    }
    if (thief) {
      want = d_want; out = (d_out & 1) != 0; prun = PS && (d_out & 2) != 0; base = d_base; slot = d_slot;
      root = d_root; tl = d_tl;
      pos = p0 + (int)((long long)w * (rank + 1) / parts);
      end = p0 + (int)((long long)w * (rank + 2) / parts);
    }
    if (lane == donor) end = p0 + (int)((long long)w / parts);
  }

  // Returns true (on every lane) once the enumeration cap is reached and the
  // search stops there (no exact total requested).
  __device__ __forceinline__ bool emit_row(bool emit, const int (&e)[KE], int last_eid) {
    const unsigned em = __ballot_sync(kFull, emit);
    if (!em) return false;
    const int leader = __ffs(em) - 1;
    unsigned long long b0 = 0;
    if (lane == leader) b0 = atomicAdd(ea.count, (unsigned long long)__popc(em));
    b0 = __shfl_sync(kFull, b0, leader);
    if (emit) {
      const unsigned long long s = b0 + (unsigned long long)__popc(em & lt);
      if (s < (unsigned long long)ea.cap) {
        int *row = ea.rows + s * K;
#pragma unroll
        for (int q = 0; q < K - 1; q++) row[q] = __ldg(g.euid + e[q < KE ? q : 0]);
        row[K - 1] = __ldg(g.euid + last_eid);
      }
      if (!ea.exact_total && s + 1 >= (unsigned long long)ea.cap) atomicExch(ea.stop, 1);
    }
    return !ea.exact_total && b0 + (unsigned long long)__popc(em) >= (unsigned long long)ea.cap;
  }
};

// Persistent search: warps claim root tiles from one work queue covering
// every query of the launch, switch their per-warp query copy when a tile
// belongs to another query, and add each query's count to counts[q].
template <int K, bool ENUM, bool EXACT, bool PS, bool CS>
__global__ void __launch_bounds__(kBlock, min_blocks(K))
search_kernel(const GraphView g, const __grid_constant__ QueryDesc q0, const LaunchArgs la,
              const __grid_constant__ EnumArgs ea) {
  extern __shared__ int4 dyn_smem[];
  WarpSmem<K> *smem = reinterpret_cast<WarpSmem<K> *>(dyn_smem);
  const int lane = threadIdx.x & 31;
  WarpSmem<K> &sm = smem[threadIdx.x >> 5];
  if (lane < K) sm.nb[lane] = 0;
  if (lane == 0) { sm.halt = 0; sm.cur_q = 0; }
  __syncwarp();
  Searcher<K, ENUM, EXACT, PS, CS> S(g, sm.q.plan, ea, la, sm, lane);
  int cur_q = -1;
  auto flush = [&]() {
    if (cur_q >= 0) {
      if (!ENUM) {
        unsigned long long c = S.cnt;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(kFull, c, o);
        if (lane == 0 && c) atomicAdd(la.counts + cur_q, c);
        S.cnt = 0;
      }
      if (la.limit) S.meter_add();
    }
  };
  while (true) {
    int t = 0;
    if (lane == 0) {
      if (ENUM && *(volatile int *)ea.stop) t = la.total_tiles;
      else t = atomicAdd(la.cursor, 1);
    }
    t = __shfl_sync(kFull, t, 0);
    if (t >= la.total_tiles) break;
    // query of this tile
    int q = 0;
    if (la.table != nullptr && la.nq > 1) {
      if (lane == 0) {
        int lo = 0, hi = la.nq;  // last query with tile_beg <= t
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (__ldg(&la.table[mid].tile_beg) <= t) lo = mid; else hi = mid;
        }
        q = lo;
      }
      q = __shfl_sync(kFull, q, 0);
    }
    if (q != cur_q) {
      flush();
      // a query table in device memory when given (batches; replayable in a
      // CUDA graph), else the single query passed by value
      const int *src = (la.table != nullptr) ? reinterpret_cast<const int *>(la.table + q)
                                             : reinterpret_cast<const int *>(&q0);
      constexpr int W = sizeof(QueryDesc) / sizeof(int);
      int *dst = reinterpret_cast<int *>(&sm.q);
      for (int i = lane; i < W; i += 32) dst[i] = src[i];
      if (lane == 0) sm.cur_q = q;
      __syncwarp();
      S.set_query(sm.q);
      cur_q = q;
    }
    if (la.limit) {
      // a query past its limit: skip its remaining tiles
      int over = 0;
      if (lane == 0) over = *(volatile unsigned long long *)(la.meter + q) > la.limit;
      if (__shfl_sync(kFull, over, 0)) continue;
    }
    const int rb = sm.q.root_beg + (t - sm.q.tile_beg) * la.tile_roots;
    const int re = min(rb + la.tile_roots, sm.q.root_end);
    const int delta = sm.q.delta;
    // the list that bounds each root's window (the last motif edge's list
    // at a root node): 0 / 1 in-list of root node 0 / 1, 2 / 3 out-list of
    // root node 0 / 1, -1 none
    int side = -1;
    if (EVX_ROOT_BOUND && S.kr() >= 3 && !(S.qf & kQNoBound)) {
      const int wl = sm.q.plan.info[S.kr() - 2];
      const int a = plan_a(wl), b = plan_b(wl);
      side = b <= 1 ? b : (a <= 1 ? 2 + a : -1);
    }
    for (int b0 = rb; b0 < re;) {
      // The roots of the next batch, packed in edge order until it holds
      // 32 or the tile ends: a root is an edge that is not a self-loop
      // (with constraints: that passes its edge predicate and node
      // predicates 0 and 1) and whose bounding list holds an entry inside
      // its window.
      int n = 0;
      while (n < 32 && b0 < re && (EVX_ROOT_PACK || n == 0)) {
        const int r = b0 + lane;
        bool ok = false;
        int4 ed = make_int4(0, 0, 0, 0);
        int tlr = 0;
        if (r < re) {
          ed = __ldg(g.edges + r);
          ok = ed.x != ed.y;
          if constexpr (CS) {
            if (ok && la.cons.edge_ok) ok = __ldg(la.cons.edge_ok + r) != 0;
            if (ok && la.cons.node_ok)
              ok = ((__ldg(la.cons.node_ok + ed.x) & 1) != 0) && ((__ldg(la.cons.node_ok + ed.y) & 2) != 0);
          }
          tlr = ed.z + delta;
          if (ok && side >= 0) {
            const int4 rg = __ldg(g.node_rng + ((side & 1) ? ed.y : ed.x));
            int st, hi;
            const int4 *lst;
            if (side < 2) {
              lst = g.in_rec; hi = rg.w;
              st = side == 0 ? __ldg(g.cross_in + r) : __ldg(g.inpos + r) + 1;
            } else {
              lst = g.out_rec; hi = rg.y;
              st = side == 2 ? ed.w + 1 : __ldg(g.cross_out + r);
            }
            const int nb = list_first_t_after(lst, st, min(hi, st + EVX_BOUND_MAX + 1), tlr) - st;
            if (nb == 0) ok = false;
            else if (nb <= EVX_BOUND_MAX) tlr = ld_t(lst + st + nb - 1);
          }
        }
        const unsigned bm = __ballot_sync(kFull, ok);
        const int rank = __popc(bm & S.lt), room = 32 - n;
        int adv = min(32, re - b0), take = __popc(bm);
        if (take > room) {
          // the batch fills at the room-th passing root: resume after it
          adv = __ffs(__ballot_sync(kFull, ok && rank == room - 1));
          take = room;
        }
        if (ok && rank < room) sm.root[n + rank] = make_int4(ed.x, ed.y, tlr, r);
        n += take;
        b0 += adv;
      }
      const bool has = lane < n;
      __syncwarp();
      if (!ENUM && S.kr() == 2 && (S.qf & kQInlineLast)) {
        // the only searched edge closes on the root's endpoints
        if (has) {
          const int4 rt = sm.root[lane];
          const int w = sm.q.plan.info[0];
          const int ia = plan_a(w) == 0 ? rt.x : rt.y, ib = plan_b(w) == 0 ? rt.x : rt.y;
          const int2 f = pair_find(g, ia, ib);
          const int key = S.strict_() ? rt.z - delta : rt.w;
          S.cnt += (unsigned long long)pair_window(g, f.x, f.y, key, rt.z, S.strict_());
        }
      } else {
        S.template level<0>(has, lane, 32);
      }
      __syncwarp();
      if (sm.halt) {
        // stopped inside this batch of roots: leave the tile (count mode);
        // enumeration also stops claiming tiles through ea.stop
        __syncwarp();
        if (lane == 0) sm.halt = 0;
        __syncwarp();
        break;
      }
      if (ENUM && *(volatile int *)ea.stop) break;
    }
  }
  flush();
}

// The shared-memory attribute belongs to the function on the current
// device, so it is set once per device (bit d of the mask: device d).
template <int K, bool ENUM, bool EXACT, bool PS, bool CS>
int setup_k() {
  static std::atomic<unsigned long long> done{0ull};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  const unsigned long long bit = dev < 64 ? (1ull << dev) : 0ull;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return 0;
  e = cudaFuncSetAttribute(search_kernel<K, ENUM, EXACT, PS, CS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(kWarps * sizeof(WarpSmem<K>)));
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
#ifdef EVX_CARVEOUT
  e = cudaFuncSetAttribute(search_kernel<K, ENUM, EXACT, PS, CS>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           EVX_CARVEOUT);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(carveout)");
#endif
  done.fetch_or(bit, std::memory_order_release);
  return 0;
}

template <int K, bool ENUM, bool EXACT, bool PS, bool CS>
int launch_k(const GraphView &g, const QueryDesc &q0, const LaunchArgs &la, const EnumArgs &ea, int grid,
             cudaStream_t s) {
  int rc = setup_k<K, ENUM, EXACT, PS, CS>();
  if (rc) return rc;
  search_kernel<K, ENUM, EXACT, PS, CS><<<grid, kBlock, kWarps * sizeof(WarpSmem<K>), s>>>(g, q0, la, ea);
  return 0;
}

template <int K, bool ENUM, bool EXACT, bool PS, bool CS>
int occ_k(int *bps) {
  int rc = setup_k<K, ENUM, EXACT, PS, CS>();
  if (rc) return rc;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, search_kernel<K, ENUM, EXACT, PS, CS>, kBlock,
                                                                kWarps * sizeof(WarpSmem<K>));
  return e == cudaSuccess ? 0 : cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
}

// Single-query launch description from the worker's SearchArgs.
QueryDesc single_query(const MotifPlan &plan, const SearchArgs &args) {
  QueryDesc q;
  memset(&q, 0, sizeof(q));
  q.plan = plan;
  q.root_beg = args.root_beg;
  q.root_end = args.root_end;
  q.delta = args.delta;
  q.flags = (args.strict_ts ? kQStrict : 0) | args.tail_flags;
  q.steal_interval = args.steal_interval;
  q.min_split = args.min_split;
  q.tile_beg = 0;
  return q;
}

constexpr int kSingleTileRoots = 64;

}  // namespace

// single-query launches: exact motif size, count or enumerate, with or
// without the pair-run walk (PS: compiled out where no level needs it), and
// the constrained variant (CS: node / edge predicates and temporal gaps,
// always with the walk)
#define EVX_K_CASE(FN, KK, ...)                                                      \
  case KK:                                                                           \
    if (cs) return enumerate ? FN<KK, true, true, true, true>(__VA_ARGS__)            \
                             : FN<KK, false, true, true, true>(__VA_ARGS__);          \
    if (enumerate) return ps ? FN<KK, true, true, true, false>(__VA_ARGS__) : FN<KK, true, true, false, false>(__VA_ARGS__); \
    return ps ? FN<KK, false, true, true, false>(__VA_ARGS__) : FN<KK, false, true, false, false>(__VA_ARGS__);
#define EVX_K_DISPATCH(FN, ...)                                        \
  switch (k) {                                                         \
    EVX_K_CASE(FN, 2, __VA_ARGS__)                                     \
    EVX_K_CASE(FN, 3, __VA_ARGS__)                                     \
    EVX_K_CASE(FN, 4, __VA_ARGS__)                                     \
    EVX_K_CASE(FN, 5, __VA_ARGS__)                                     \
    EVX_K_CASE(FN, 6, __VA_ARGS__)                                     \
    EVX_K_CASE(FN, 7, __VA_ARGS__)                                     \
    EVX_K_CASE(FN, 8, __VA_ARGS__)                                     \
    default: return fail(EVX_ERR_INVALID, "motif edge count out of range");          \
  }

// Whether a query walks a pair run at some level: an edge between two nodes
// mapped before it that is scanned (every level before the last; the last
// one only when enumerating: a counted closing last edge takes range
// arithmetic instead).
bool plan_pair_scan(const MotifPlan &plan, int qflags, bool enumerate) {
  if (!(qflags & kQPairScan)) return false;
  for (int l = 0; l <= plan.k - 2; l++) {
    if (plan_kind(plan.info[l]) != 2) continue;
    if (l < plan.k - 2 || enumerate) return true;
  }
  return false;
}

int launch_search(const GraphView &g, const MotifPlan &plan, const SearchArgs &args, int grid, int block,
                  cudaStream_t stream) {
  (void)block;
  const int k = plan.k;
  const bool enumerate = args.enumerate != 0;
  const QueryDesc q0 = single_query(plan, args);
  LaunchArgs la{};
  la.table = nullptr;
  la.nq = 1;
  la.tile_roots = kSingleTileRoots;
  const int n = args.root_end - args.root_beg;
  la.total_tiles = n > 0 ? (n + kSingleTileRoots - 1) / kSingleTileRoots : 0;
  la.cursor = args.cursor;
  la.counts = args.count;
  la.limit = args.limit;
  la.meter = args.meter;
  EnumArgs ea;
  ea.rows = args.rows;
  ea.cap = args.cap;
  ea.exact_total = args.exact_total;
  ea.stop = args.stop;
  ea.count = args.count;
  const bool ps = plan_pair_scan(plan, q0.flags, enumerate);
  la.cons = args.cons;
  const bool cs = cons_any(args.cons);
  EVX_K_DISPATCH(launch_k, g, q0, la, ea, grid, stream)
}

int launch_table(const GraphView &g, const QueryDesc &q0, const LaunchArgs &la, int k, bool ps, int grid,
                 cudaStream_t stream) {
  const bool enumerate = false, cs = false;
  EnumArgs ea;
  memset(&ea, 0, sizeof(ea));
  EVX_K_DISPATCH(launch_k, g, q0, la, ea, grid, stream)
}

int search_occupancy(int k, bool enumerate, bool ps, bool cs, int block, int *blocks_per_sm) {
  (void)block;
  EVX_K_DISPATCH(occ_k, blocks_per_sm)
}

int table_occupancy(int k, bool ps, int *blocks_per_sm) {
  const bool enumerate = false, cs = false;
  EVX_K_DISPATCH(occ_k, blocks_per_sm)
}

int search_block_size() { return kBlock; }

}  // namespace evx
