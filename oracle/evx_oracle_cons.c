/*
 * evx_oracle_cons.c -- CPU restatement of the reference's constrained search
 * (node / edge predicates, temporal gaps, anti-edges, filters).
 *
 * TEST INFRASTRUCTURE ONLY, like evx_oracle.c: tests and the fixture script
 * call it as the checker; the product never links it.
 *
 * Semantics restated from the code the reference generates per query
 * (system/tmine/Query.py:39-310, system/tmine/KernelGen.py:288-336,467-534,
 * system/templates/common/{nextMatchInTask,structuralConstraint,
 * lookAtMatchRes,findMatch,nextLevel,mapFirst}.snp,
 * system/templates/dispatch/processFirstEdge.snp):
 *  - root e_0 needs u != v, node predicate 0 on u, node predicate 1 on v
 *    and the edge predicate (processFirstEdge.snp:1-4);
 *  - motif edge j >= 1 scans the list that resolveMi.snp picks, from the
 *    first entry after the previous REAL edge (antiEdgePrev,
 *    Query.py:64-73, KernelGen.py:479-497) up to the window end tl_j;
 *  - tl_1 = t(e_0) + temporal[0] (mapFirst.snp:4, KernelGen.py:472-473)
 *    when a temporal list is given, tl_j = min(t(prev real) + temporal[j-1],
 *    t(e_0) + delta) for j >= 2 (KernelGen.py:475-476); tl_j = t(e_0) +
 *    delta for every j without one.  For k >= 3 the first window is also
 *    capped by t(e_0) + delta on every backtrack, which cannot change a
 *    count: a later edge must lie inside t(e_0) + delta and after e_1;
 *  - a candidate passes when its mapped endpoint matches, or its new
 *    endpoint differs from every mapped node and passes the node predicate
 *    of its motif node, and its edge passes the edge predicate
 *    (structuralConstraint.snp, Query.py:218-223,262-267);
 *  - an anti-edge level drops the partial match when any candidate passes,
 *    else continues with nothing mapped (lookAtMatchRes.snp:1-21);
 *  - a complete match counts when the filter holds (findMatch.snp:1-8).
 */
#include <stdint.h>
#include <string.h>

#include "../include/everest_b200.h"

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------ expression programs -- */
int64_t oracle_prog_eval(const evx_program *p, const int64_t *vars) {
  int64_t st[EVX_PROG_STACK + 2];
  int sp = 0;
  if (p->len == 0) return 1;
  for (int i = 0; i < p->len; i++) {
    const int op = p->op[i] & 0x7f;
    const int w = (p->op[i] & EVX_OP_WRAP32) != 0;
    int64_t r;
    if (op == EVX_OP_CONST) { st[sp++] = p->arg[i]; continue; }
    if (op == EVX_OP_VAR) { st[sp++] = vars[p->arg[i]]; continue; }
    if (op == EVX_OP_NEG || op == EVX_OP_NOT || op == EVX_OP_BNOT) {
      const int64_t a = st[--sp];
      r = op == EVX_OP_NEG ? (int64_t)(0 - (uint64_t)a) : op == EVX_OP_NOT ? (a == 0) : ~a;
    } else if (op == EVX_OP_COND) {
      const int64_t b = st[--sp], a = st[--sp], c = st[--sp];
      r = c ? a : b;
    } else {
      const int64_t b = st[--sp], a = st[--sp];
      switch (op) {
        case EVX_OP_ADD: r = (int64_t)((uint64_t)a + (uint64_t)b); break;
        case EVX_OP_SUB: r = (int64_t)((uint64_t)a - (uint64_t)b); break;
        case EVX_OP_MUL: r = (int64_t)((uint64_t)a * (uint64_t)b); break;
        case EVX_OP_DIV:
          r = b == 0 ? 0 : (b == -1 ? (int64_t)(0 - (uint64_t)a) : a / b);
          break;
        case EVX_OP_MOD: r = (b == 0 || b == -1) ? 0 : a % b; break;
        case EVX_OP_SHL: r = (int64_t)((uint64_t)a << (b & (w ? 31 : 63))); break;
        case EVX_OP_SHR: r = a >> (b & (w ? 31 : 63)); break;
        case EVX_OP_LT: r = a < b; break;
        case EVX_OP_LE: r = a <= b; break;
        case EVX_OP_GT: r = a > b; break;
        case EVX_OP_GE: r = a >= b; break;
        case EVX_OP_EQ: r = a == b; break;
        case EVX_OP_NE: r = a != b; break;
        case EVX_OP_BAND: r = a & b; break;
        case EVX_OP_BXOR: r = a ^ b; break;
        case EVX_OP_BOR: r = a | b; break;
        case EVX_OP_LAND: r = (a != 0) && (b != 0); break;
        case EVX_OP_LOR: r = (a != 0) || (b != 0); break;
        default: return 0;
      }
    }
    if (w) r = (int64_t)(int32_t)(uint32_t)(uint64_t)r;
    st[sp++] = r;
  }
  return st[sp - 1];
}

/* ------------------------------------------------------------- search -- */
typedef struct {
  const int *u, *v, *t;
  const int *out_off, *out_eid, *in_off, *in_eid;
  const int *node_feat, *edge_feat;
  int k, delta;
  const int *mu, *mv;
  int nmapped[EVX_MAX_MOTIF_EDGES];
  int prev_real[EVX_MAX_MOTIF_EDGES];
  const evx_constraints *c;
} cons_ctx;

typedef struct {
  uint64_t count;
  uint64_t roots, r_reads, candidates;  /* the algorithmic-bytes counters of evx_oracle.c */
  int m[EVX_MAX_MOTIF_NODES + 1];
  int e[EVX_MAX_MOTIF_EDGES];
  int *rows;
  int64_t cap, nrows;
} cons_state;

static int node_ok(const cons_ctx *x, int node, int a) {
  const evx_constraints *c = x->c;
  if (c->node_mode == 0) return 1;
  const evx_program *p = &c->node[c->node_mode == 1 ? 0 : a];
  int64_t f = x->node_feat[node];
  return oracle_prog_eval(p, &f) != 0;
}

static int edge_ok(const cons_ctx *x, int e) {
  if (!x->c->has_edge) return 1;
  int64_t f = x->edge_feat[e];
  return oracle_prog_eval(&x->c->edge, &f) != 0;
}

static int filter_ok(const cons_ctx *x, const cons_state *s) {
  if (!x->c->has_filter) return 1;
  int64_t vars[EVX_MAX_MOTIF_EDGES];
  for (int q = 0; q < x->k; q++)
    vars[q] = ((x->c->anti_mask >> q) & 1) ? 0 : x->edge_feat[s->e[q]];
  return oracle_prog_eval(&x->c->filter, vars) != 0;
}

static int first_after(const int *lst, int beg, int end, int prev) {
  while (beg < end) {
    int mid = beg + (end - beg) / 2;
    if (lst[mid] > prev) end = mid; else beg = mid + 1;
  }
  return beg;
}

static void cdfs(const cons_ctx *x, cons_state *s, int j) {
  const evx_constraints *c = x->c;
  const int a = x->mu[j], b = x->mv[j];
  const int nm = x->nmapped[j];
  const int pr = s->e[x->prev_real[j]];
  const int t0 = x->t[s->e[0]];
  int tl;
  if (c->has_temporal) {
    const int64_t g = (int64_t)x->t[pr] + c->temporal[j - 1];
    tl = (int)g;
    if (j >= 2 && (int64_t)t0 + x->delta < g) tl = t0 + x->delta;
  } else {
    tl = t0 + x->delta;
  }
  const int *lst;
  int lo, hi, want = -1, other_is_v;
  if (a < nm && b < nm) {
    const int ma = s->m[a], mb = s->m[b];
    const int ib = x->in_off[mb], ie = x->in_off[mb + 1];
    const int ob = x->out_off[ma], oe = x->out_off[ma + 1];
    s->r_reads += 2;
    if (ie - ib < oe - ob) { lst = x->in_eid; lo = ib; hi = ie; want = ma; other_is_v = 0; }
    else { lst = x->out_eid; lo = ob; hi = oe; want = mb; other_is_v = 1; }
  } else if (b >= nm) {
    lst = x->out_eid; lo = x->out_off[s->m[a]]; hi = x->out_off[s->m[a] + 1]; other_is_v = 1;
    s->r_reads += 1;
  } else {
    lst = x->in_eid; lo = x->in_off[s->m[b]]; hi = x->in_off[s->m[b] + 1]; other_is_v = 0;
    s->r_reads += 1;
  }
  lo = first_after(lst, lo, hi, pr);
  const int anti = (c->anti_mask >> j) & 1;
  const int last = (j == x->k - 1);
  for (int p = lo; p < hi; p++) {
    const int ce = lst[p];
    s->candidates++;
    if (x->t[ce] > tl) break;
    const int node = other_is_v ? x->v[ce] : x->u[ce];
    int ok;
    if (want >= 0) {
      ok = (node == want);
    } else {
      ok = 1;
      for (int q = 0; q < nm; q++) if (s->m[q] == node) { ok = 0; break; }
      if (ok) ok = node_ok(x, node, nm);
    }
    if (!ok || !edge_ok(x, ce)) continue;
    if (anti) return;  /* the edge that must not exist does */
    s->e[j] = ce;
    if (last) {
      if (filter_ok(x, s)) {
        s->count++;
        if (s->rows && s->nrows < s->cap) {
          int *row = s->rows + s->nrows * x->k;
          for (int q = 0; q < x->k; q++) row[q] = s->e[q];
        }
        s->nrows++;
      }
    } else {
      if (want < 0) s->m[nm] = node;
      cdfs(x, s, j + 1);
    }
  }
  if (anti) {  /* none found: go on with this edge unmatched */
    s->e[j] = -1;
    cdfs(x, s, j + 1);
  }
}

static void cons_root(const cons_ctx *x, cons_state *s, int64_t r) {
  s->roots++;
  if (x->u[r] == x->v[r]) return;
  if (!node_ok(x, x->u[r], 0) || !node_ok(x, x->v[r], 1) || !edge_ok(x, (int)r)) return;
  s->m[0] = x->u[r];
  s->m[1] = x->v[r];
  s->e[0] = (int)r;
  cdfs(x, s, 1);
}

static int cons_setup(cons_ctx *x, const int *u, const int *v, const int *t,
                      const int *out_off, const int *out_eid, const int *in_off, const int *in_eid,
                      const int *node_feat, const int *edge_feat,
                      int k, const int *mu, const int *mv, int delta, const evx_constraints *c) {
  memset(x, 0, sizeof(*x));
  if (k < 2 || k > EVX_MAX_MOTIF_EDGES || mu[0] != 0 || mv[0] != 1) return -1;
  x->u = u; x->v = v; x->t = t;
  x->out_off = out_off; x->out_eid = out_eid; x->in_off = in_off; x->in_eid = in_eid;
  x->node_feat = node_feat; x->edge_feat = edge_feat;
  x->k = k; x->delta = delta; x->mu = mu; x->mv = mv; x->c = c;
  int nm = 2;
  for (int j = 1; j < k; j++) {
    x->nmapped[j] = nm;
    const int an = mu[j] >= nm, bn = mv[j] >= nm;
    if (mu[j] == mv[j] || (an && bn)) return -1;
    if (an || bn) nm++;
    int p = j - 1;
    while (p > 0 && ((c->anti_mask >> p) & 1)) p--;
    x->prev_real[j] = p;
  }
  if ((c->node_mode && !node_feat) || ((c->has_edge || c->has_filter) && !edge_feat)) return -1;
  return 0;
}

/* Constrained count over roots [root_beg, root_end).  stats (may be NULL)
 * receives {roots, r_reads, candidates} as evx_oracle.c counts them. */
int oracle_count_constrained(const int *u, const int *v, const int *t,
                             const int *out_off, const int *out_eid,
                             const int *in_off, const int *in_eid,
                             const int *node_feat, const int *edge_feat,
                             int k, const int *mu, const int *mv, int delta,
                             const evx_constraints *c, int64_t root_beg, int64_t root_end,
                             int nthreads, uint64_t *count_out, uint64_t *stats) {
  cons_ctx x;
  if (cons_setup(&x, u, v, t, out_off, out_eid, in_off, in_eid, node_feat, edge_feat, k, mu, mv,
                 delta, c))
    return -1;
  uint64_t total = 0, roots = 0, rr = 0, cand = 0;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads) reduction(+ : total, roots, rr, cand)
#endif
  for (int64_t r = root_beg; r < root_end; r++) {
    cons_state s;
    memset(&s, 0, sizeof(s));
    cons_root(&x, &s, r);
    total += s.count;
    roots += s.roots;
    rr += s.r_reads;
    cand += s.candidates;
  }
  (void)nthreads;
  *count_out = total;
  if (stats) {
    stats[0] = roots;
    stats[1] = rr;
    stats[2] = cand;
  }
  return 0;
}

/* Constrained enumeration (serial): up to cap rows of k sorted-edge ids. */
int oracle_enumerate_constrained(const int *u, const int *v, const int *t,
                                 const int *out_off, const int *out_eid,
                                 const int *in_off, const int *in_eid,
                                 const int *node_feat, const int *edge_feat,
                                 int k, const int *mu, const int *mv, int delta,
                                 const evx_constraints *c, int64_t root_beg, int64_t root_end,
                                 int *rows, int64_t cap, uint64_t *total) {
  cons_ctx x;
  if (cons_setup(&x, u, v, t, out_off, out_eid, in_off, in_eid, node_feat, edge_feat, k, mu, mv,
                 delta, c))
    return -1;
  cons_state s;
  memset(&s, 0, sizeof(s));
  s.rows = rows;
  s.cap = cap;
  for (int64_t r = root_beg; r < root_end; r++) cons_root(&x, &s, r);
  *total = s.count;
  return 0;
}
