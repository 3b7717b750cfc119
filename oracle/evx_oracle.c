/*
 * evx_oracle.c -- CPU restatement of the reference's temporal-motif search.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load this library, and only as the checker or
 * as the timed CPU port.  The product path (everest_b200) never links it.
 *
 * Semantics restated (reference file:line):
 *  - Edges are indexed by their position after a stable sort on t
 *    (src/core/cpu/data.cc:246-248); the inputs here are already in that
 *    order, so edge id == array index.
 *  - Per-node out/in edge-id lists are ascending in edge id
 *    (src/core/gpu/data.cu:242-271: stable_sort_by_key on the endpoint).
 *  - A root is every edge id in [beg, end) with u != v
 *    (system/templates/dispatch/processFirstEdge.snp:1); the default job is
 *    [0, E-k+1) (src/core/cpu/data.cc:452-457).
 *  - The window is t(e_j) <= t(e_0) + delta, inclusive, computed in int
 *    (system/templates/common/mapFirst.snp:3,
 *     system/templates/common/nextMatchInTask.snp:6).
 *  - Motif edge j >= 1 scans the out-list of the mapped source when its
 *    target is new, the in-list of the mapped target when its source is new,
 *    and the shorter of in(target)/out(source) when both are mapped (ties go
 *    to the out-list) (src/core/cpu/data.cc:423-446,
 *    system/templates/common/resolveMi.snp:1-28).
 *  - The scan starts at the first list entry whose edge id is greater than
 *    the previous level's edge id (system/templates/funcs/reduceEarlyIdx.snp)
 *    and stops at the first entry with t > tl
 *    (system/templates/common/nextMatchInTask.snp:1-21).
 *  - A new node must differ from every node mapped so far; a mapped node
 *    must equal its image (system/tmine/KernelGen.py:419-451,
 *    system/templates/common/structuralConstraint.snp).
 *  - Enumeration rows are the original line ids (Euid) of e_0..e_{k-1}
 *    (system/tmine/KernelGen.py:505-524).
 *
 * Instrumentation (the algorithmic-bytes model of the serial semantics):
 *  roots      = roots tried (every id in the job range),
 *  r_reads    = CSR offset pairs read per list opening (2 for a closing edge),
 *  candidates = inner-loop iterations of the candidate scan, including the
 *               one terminating t > tl probe of each list, excluding binary
 *               search probes,
 *  list_opens = list openings.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_MAXK 16
#define ORACLE_MAXN 17

typedef struct {
  uint64_t roots, r_reads, candidates, list_opens, matches;
} oracle_stats;

typedef struct {
  const int *u, *v, *t;
  const int *out_off, *out_eid, *in_off, *in_eid;
  int k;
  const int *mu, *mv;
  int nmapped[ORACLE_MAXK]; /* nodes mapped before motif edge j */
  int strict_ts;
} oracle_ctx;

/* ------------------------------------------------------------ CSR build -- */
/* Stable counting sort of edge ids by endpoint: lists ascend in edge id. */
int oracle_build_csr(int64_t E, int V, const int *u, const int *v,
                     int *out_off, int *out_eid, int *in_off, int *in_eid) {
  memset(out_off, 0, sizeof(int) * (size_t)(V + 1));
  memset(in_off, 0, sizeof(int) * (size_t)(V + 1));
  for (int64_t i = 0; i < E; i++) {
    if (u[i] < 0 || u[i] >= V || v[i] < 0 || v[i] >= V) return -1;
    out_off[u[i] + 1]++;
    in_off[v[i] + 1]++;
  }
  for (int x = 0; x < V; x++) {
    out_off[x + 1] += out_off[x];
    in_off[x + 1] += in_off[x];
  }
  int *oc = (int *)malloc(sizeof(int) * (size_t)V);
  int *ic = (int *)malloc(sizeof(int) * (size_t)V);
  if (!oc || !ic) { free(oc); free(ic); return -2; }
  memcpy(oc, out_off, sizeof(int) * (size_t)V);
  memcpy(ic, in_off, sizeof(int) * (size_t)V);
  for (int64_t i = 0; i < E; i++) {
    out_eid[oc[u[i]]++] = (int)i;
    in_eid[ic[v[i]]++] = (int)i;
  }
  free(oc);
  free(ic);
  return 0;
}

/* ---------------------------------------------------------- motif rules -- */
/* Nodes mapped before each motif edge; -1 if a later edge touches no mapped
 * node or is a self-loop (the reference's implicit precondition,
 * src/core/cpu/data.cc:416-446). Edges must already be relabeled by first
 * appearance with edge 0 = (0, 1). */
int oracle_motif_nmapped(int k, const int *mu, const int *mv, int *nmapped) {
  if (k < 2 || k > ORACLE_MAXK) return -1;
  if (mu[0] != 0 || mv[0] != 1) return -1;
  int nm = 2;
  nmapped[0] = 0;
  for (int j = 1; j < k; j++) {
    nmapped[j] = nm;
    int a = mu[j], b = mv[j];
    if (a == b) return -1;
    int an = a >= nm, bn = b >= nm;
    if (an && bn) return -1;
    if (an) { if (a != nm) return -1; nm++; }
    if (bn) { if (b != nm) return -1; nm++; }
  }
  if (nm > ORACLE_MAXN) return -1;
  return nm;
}

/* first position in lst[beg, end) whose value is > prev */
static int first_after(const int *lst, int beg, int end, int prev) {
  while (beg < end) {
    int mid = beg + (end - beg) / 2;
    if (lst[mid] > prev) end = mid; else beg = mid + 1;
  }
  return beg;
}

typedef struct {
  uint64_t count;
  oracle_stats st;
  int m[ORACLE_MAXN];
  int e[ORACLE_MAXK];
  int tl;
  /* enumeration sink */
  int *rows;
  int64_t cap, nrows;
} oracle_state;

static void dfs(const oracle_ctx *c, oracle_state *s, int j) {
  const int a = c->mu[j], b = c->mv[j];
  const int nm = c->nmapped[j];
  const int prev = s->e[j - 1];
  const int *lst;
  int lo, hi;
  int want = -1;          /* mapped image to match, or -1 for "new node" */
  int other_is_v;         /* candidate's checked endpoint: v (out-list) or u (in-list) */
  if (a < nm && b < nm) { /* closing edge: both endpoints mapped */
    int ma = s->m[a], mb = s->m[b];
    int ib = c->in_off[mb], ie = c->in_off[mb + 1];
    int ob = c->out_off[ma], oe = c->out_off[ma + 1];
    s->st.r_reads += 2;
    if (ie - ib < oe - ob) { lst = c->in_eid; lo = ib; hi = ie; want = ma; other_is_v = 0; }
    else { lst = c->out_eid; lo = ob; hi = oe; want = mb; other_is_v = 1; }
  } else if (b >= nm) {   /* new target: out-list of the mapped source */
    int ma = s->m[a];
    lst = c->out_eid; lo = c->out_off[ma]; hi = c->out_off[ma + 1]; other_is_v = 1;
    s->st.r_reads += 1;
  } else {                /* new source: in-list of the mapped target */
    int mb = s->m[b];
    lst = c->in_eid; lo = c->in_off[mb]; hi = c->in_off[mb + 1]; other_is_v = 0;
    s->st.r_reads += 1;
  }
  s->st.list_opens++;
  lo = first_after(lst, lo, hi, prev);
  const int last = (j == c->k - 1);
  for (int p = lo; p < hi; p++) {
    const int ce = lst[p];
    s->st.candidates++;
    if (c->t[ce] > s->tl) break;
    const int node = other_is_v ? c->v[ce] : c->u[ce];
    int ok;
    if (want >= 0) {
      ok = (node == want);
    } else {
      ok = 1;
      for (int q = 0; q < nm; q++) if (s->m[q] == node) { ok = 0; break; }
    }
    if (!ok) continue;
    if (c->strict_ts && !(c->t[ce] > c->t[prev])) continue;
    s->e[j] = ce;
    if (last) {
      s->count++;
      if (s->rows && s->nrows < s->cap) {
        int *row = s->rows + s->nrows * c->k;
        for (int q = 0; q < c->k; q++) row[q] = s->e[q];
      }
      s->nrows++;
    } else {
      if (want < 0) s->m[nm] = node;
      dfs(c, s, j + 1);
    }
  }
}

/* One root: the first motif edge maps (0, 1) to (u, v); self-loops are not
 * roots (system/templates/dispatch/processFirstEdge.snp:1). */
static void run_root(const oracle_ctx *c, oracle_state *s, int64_t r, int delta) {
  s->st.roots++;
  if (c->u[r] == c->v[r]) return;
  s->m[0] = c->u[r];
  s->m[1] = c->v[r];
  s->e[0] = (int)r;
  s->tl = c->t[r] + delta;
  dfs(c, s, 1);
}

static int setup_ctx(oracle_ctx *c, const int *u, const int *v, const int *t,
                     const int *out_off, const int *out_eid,
                     const int *in_off, const int *in_eid,
                     int k, const int *mu, const int *mv, int strict_ts) {
  memset(c, 0, sizeof(*c));
  c->u = u; c->v = v; c->t = t;
  c->out_off = out_off; c->out_eid = out_eid;
  c->in_off = in_off; c->in_eid = in_eid;
  c->k = k; c->mu = mu; c->mv = mv;
  c->strict_ts = strict_ts;
  return oracle_motif_nmapped(k, mu, mv, c->nmapped) < 0 ? -1 : 0;
}

/* Count matches for roots in [root_beg, root_end).  Returns 0, or -1 on a
 * bad motif.  stats may be NULL. */
int oracle_count(const int *u, const int *v, const int *t,
                 const int *out_off, const int *out_eid,
                 const int *in_off, const int *in_eid,
                 int k, const int *mu, const int *mv, int delta,
                 int64_t root_beg, int64_t root_end, int strict_ts,
                 int nthreads, uint64_t *count_out, oracle_stats *stats) {
  oracle_ctx c;
  if (setup_ctx(&c, u, v, t, out_off, out_eid, in_off, in_eid, k, mu, mv, strict_ts))
    return -1;
  uint64_t total = 0, roots = 0, rr = 0, cand = 0, opens = 0;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads) \
    reduction(+ : total, roots, rr, cand, opens)
#endif
  for (int64_t r = root_beg; r < root_end; r++) {
    oracle_state s;
    memset(&s.st, 0, sizeof(s.st));
    s.count = 0;
    s.rows = NULL; s.cap = 0; s.nrows = 0;
    run_root(&c, &s, r, delta);
    total += s.count;
    roots += s.st.roots;
    rr += s.st.r_reads;
    cand += s.st.candidates;
    opens += s.st.list_opens;
  }
  (void)nthreads;
  *count_out = total;
  if (stats) {
    stats->roots = roots;
    stats->r_reads = rr;
    stats->candidates = cand;
    stats->list_opens = opens;
    stats->matches = total;
  }
  return 0;
}

/* Per-root counts (for debugging and for splitting work by cost). */
int oracle_count_per_root(const int *u, const int *v, const int *t,
                          const int *out_off, const int *out_eid,
                          const int *in_off, const int *in_eid,
                          int k, const int *mu, const int *mv, int delta,
                          int64_t root_beg, int64_t root_end, int strict_ts,
                          uint64_t *counts, uint64_t *cands) {
  oracle_ctx c;
  if (setup_ctx(&c, u, v, t, out_off, out_eid, in_off, in_eid, k, mu, mv, strict_ts))
    return -1;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t r = root_beg; r < root_end; r++) {
    oracle_state s;
    memset(&s.st, 0, sizeof(s.st));
    s.count = 0; s.rows = NULL; s.cap = 0; s.nrows = 0;
    run_root(&c, &s, r, delta);
    counts[r - root_beg] = s.count;
    if (cands) cands[r - root_beg] = s.st.candidates;
  }
  return 0;
}

/* Enumerate matches (serial, in root order then DFS order).  Writes up to
 * cap rows of k edge ids into rows; returns the total number of matches in
 * *total.  Rows hold sorted-edge ids; the caller maps them through Euid. */
int oracle_enumerate(const int *u, const int *v, const int *t,
                     const int *out_off, const int *out_eid,
                     const int *in_off, const int *in_eid,
                     int k, const int *mu, const int *mv, int delta,
                     int64_t root_beg, int64_t root_end, int strict_ts,
                     int *rows, int64_t cap, uint64_t *total) {
  oracle_ctx c;
  if (setup_ctx(&c, u, v, t, out_off, out_eid, in_off, in_eid, k, mu, mv, strict_ts))
    return -1;
  oracle_state s;
  memset(&s, 0, sizeof(s));
  s.rows = rows;
  s.cap = cap;
  for (int64_t r = root_beg; r < root_end; r++) run_root(&c, &s, r, delta);
  *total = s.count;
  return 0;
}
