// Constrained search: node / edge predicates, temporal gaps, anti-edges and
// filters (include/everest_b200.h, "constraints").
//
// The reference compiles every constrained query into its own CUDA plugin
// (system/tmine/Query.py:135-310 renders the predicates as C functions,
// system/tmine/KernelGen.py:467-534 the temporal, anti-edge and filter code).
// Here one kernel per motif size reads the constraints as data:
//
//  - node and edge predicates are programs (postfix, int64 stack) evaluated
//    ONCE per graph node / edge by the mask kernels below into a u16 bit set
//    per node (bit a: may be motif node a) and a byte per edge, so the search
//    tests a candidate with one gather instead of running the predicate;
//  - the search is one depth-first walk per lane over the packed 16-byte
//    adjacency records {eid, other, t, pos} (the same layout as the count
//    kernel), with per-level window ends from the temporal gaps, anti-edge
//    levels that only ask "does any candidate exist", and the filter
//    program run once per complete match;
//  - idle lanes of a warp claim new roots together: one atomicAdd per warp
//    for all of them.
//
// Semantics follow the reference's generated search
// (system/templates/common/{nextMatchInTask,structuralConstraint,
// lookAtMatchRes,findMatch,nextLevel,mapFirst}.snp,
// system/templates/dispatch/processFirstEdge.snp): a root passes node
// predicates 0 and 1 and the edge predicate; motif edge j scans from the
// first entry after the previous real edge; tl_1 = t(e_0) + temporal[0],
// tl_j = min(t(previous real edge) + temporal[j-1], t(e_0) + delta) for
// j >= 2 (t(e_0) + delta throughout without a temporal list); a new node
// must pass the predicate of its motif node; an anti-edge level drops the
// partial match when any candidate passes; a complete match counts when the
// filter holds.
#include <climits>
#include <cstring>

#include "evx_internal.cuh"

namespace evx {

constexpr int kConsBlock = 128;

// ------------------------------------------------------------ programs --
// Interpreter of the program format of include/everest_b200.h.  A stack
// index outside [0, EVX_PROG_STACK) cannot occur for programs that passed
// cons_check_program; the guards keep a bad one from writing out of bounds.
template <class Var>
__device__ __forceinline__ long long prog_eval(const evx_program &p, Var var) {
  long long st[EVX_PROG_STACK];
  int sp = 0;
  const int len = p.len;
  if (len == 0) return 1;
  for (int i = 0; i < len; i++) {
    const int opw = p.op[i];
    const int op = opw & 0x7f;
    const bool w = (opw & EVX_OP_WRAP32) != 0;
    long long r;
    if (op == EVX_OP_CONST || op == EVX_OP_VAR) {
      if (sp >= EVX_PROG_STACK) return 0;
      st[sp++] = op == EVX_OP_CONST ? p.arg[i] : var((int)p.arg[i]);
      continue;
    }
    if (op == EVX_OP_NEG || op == EVX_OP_NOT || op == EVX_OP_BNOT) {
      if (sp < 1) return 0;
      const long long a = st[--sp];
      r = op == EVX_OP_NEG ? (long long)(0ull - (unsigned long long)a) : op == EVX_OP_NOT ? (a == 0) : ~a;
    } else if (op == EVX_OP_COND) {
      if (sp < 3) return 0;
      const long long b = st[--sp], a = st[--sp], c = st[--sp];
      r = c ? a : b;
    } else {
      if (sp < 2) return 0;
      const long long b = st[--sp], a = st[--sp];
      const unsigned long long ua = (unsigned long long)a, ub = (unsigned long long)b;
      switch (op) {
        case EVX_OP_ADD: r = (long long)(ua + ub); break;
        case EVX_OP_SUB: r = (long long)(ua - ub); break;
        case EVX_OP_MUL: r = (long long)(ua * ub); break;
        case EVX_OP_DIV: r = b == 0 ? 0 : (b == -1 ? (long long)(0ull - ua) : a / b); break;
        case EVX_OP_MOD: r = (b == 0 || b == -1) ? 0 : a % b; break;
        case EVX_OP_SHL: r = (long long)(ua << (b & (w ? 31 : 63))); break;
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
    if (w) r = (long long)(int)(unsigned)(unsigned long long)r;
    st[sp++] = r;
  }
  return sp > 0 ? st[sp - 1] : 0;
}

int cons_check_program(const evx_program &p, int num_vars, const char *what) {
  if (p.len < 0 || p.len > EVX_PROG_MAX)
    return fail(EVX_ERR_INVALID, std::string(what) + ": program length out of range");
  int sp = 0;
  for (int i = 0; i < p.len; i++) {
    const int op = p.op[i] & 0x7f;
    if ((p.op[i] & ~(0x7f | EVX_OP_WRAP32)) != 0 || op < EVX_OP_CONST || op > EVX_OP_COND)
      return fail(EVX_ERR_INVALID, std::string(what) + ": bad opcode");
    int need = 2, push = 1;
    if (op == EVX_OP_CONST || op == EVX_OP_VAR) need = 0;
    else if (op == EVX_OP_NEG || op == EVX_OP_NOT || op == EVX_OP_BNOT) need = 1;
    else if (op == EVX_OP_COND) need = 3;
    if (op == EVX_OP_VAR && (p.arg[i] < 0 || p.arg[i] >= num_vars))
      return fail(EVX_ERR_INVALID, std::string(what) + ": variable index out of range");
    if (sp < need) return fail(EVX_ERR_INVALID, std::string(what) + ": stack underflow");
    sp = sp - need + push;
    if (sp > EVX_PROG_STACK) return fail(EVX_ERR_INVALID, std::string(what) + ": stack too deep");
  }
  if (p.len > 0 && sp != 1) return fail(EVX_ERR_INVALID, std::string(what) + ": does not leave one value");
  return EVX_OK;
}

// --------------------------------------------------------------- masks --
__global__ void __launch_bounds__(256) cons_node_mask_kernel(const int *__restrict__ feat, int V, int n,
                                                             const __grid_constant__ evx_constraints c,
                                                             unsigned short *__restrict__ out) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < V; x += gridDim.x * blockDim.x) {
    const long long f = __ldg(feat + x);
    auto var = [&](int) { return f; };
    unsigned m = 0;
    if (c.node_mode == 1) {
      if (prog_eval(c.node[0], var)) m = (1u << n) - 1;
    } else {
      for (int a = 0; a < n; a++)
        if (prog_eval(c.node[a], var)) m |= 1u << a;
    }
    out[x] = (unsigned short)m;
  }
}

__global__ void __launch_bounds__(256) cons_edge_mask_kernel(const int *__restrict__ feat, int E,
                                                             const __grid_constant__ evx_program p,
                                                             unsigned char *__restrict__ out) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < E; x += gridDim.x * blockDim.x) {
    const long long f = __ldg(feat + x);
    out[x] = prog_eval(p, [&](int) { return f; }) ? 1 : 0;
  }
}

int cons_build_masks(const evx_constraints &c, int n, const int *node_feat, int V, const int *edge_feat,
                     int E, unsigned short *node_ok, unsigned char *edge_ok, int num_sms, cudaStream_t s) {
  if (c.node_mode && V > 0) {
    const int grid = (int)std::min<long long>(((long long)V + 255) / 256, 8LL * num_sms);
    cons_node_mask_kernel<<<grid, 256, 0, s>>>(node_feat, V, n, c, node_ok);
    EVX_CUDA(cudaGetLastError());
  }
  if (c.has_edge && E > 0) {
    const int grid = (int)std::min<long long>(((long long)E + 255) / 256, 8LL * num_sms);
    cons_edge_mask_kernel<<<grid, 256, 0, s>>>(edge_feat, E, c.edge, edge_ok);
    EVX_CUDA(cudaGetLastError());
  }
  return EVX_OK;
}

// -------------------------------------------------------------- search --
// first position in recs[lo, hi) whose edge id is greater than e
__device__ __forceinline__ int first_eid_after(const int4 *__restrict__ recs, int lo, int hi, int e) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&recs[mid].x) > e) hi = mid; else lo = mid + 1;
  }
  return lo;
}

// Per-lane search state of one warp, indexed [level][lane]: each lane keeps
// its own column, so the dynamically indexed levels cost shared-memory
// accesses (conflict-free: 32 lanes, 32 consecutive words) instead of a
// local-memory stack.
// Roots whose last motif edge cannot occur are dropped at the claim (0: off).
#ifndef EVX_CONS_ROOT_DROP
#define EVX_CONS_ROOT_DROP 1
#endif

template <int K>
struct ConsWarpState {
  int m[K + 1][32];             // graph node of each motif node
  int eid[K][32], et[K][32];    // matched edge and its time per motif edge (anti: none)
  int pos[K][32], endp[K][32], tlv[K][32];
};

template <int K, bool ENUM>
__global__ void __launch_bounds__(kConsBlock) cons_search_kernel(const GraphView g,
                                                                 const __grid_constant__ ConsSearch s) {
  const int lane = threadIdx.x & 31;
  __shared__ ConsWarpState<K> wst[kConsBlock / 32];
  ConsWarpState<K> &W = wst[threadIdx.x >> 5];
  auto m = [&](int i) -> int & { return W.m[i][lane]; };
  auto eid = [&](int i) -> int & { return W.eid[i][lane]; };
  auto et = [&](int i) -> int & { return W.et[i][lane]; };
  auto pos = [&](int i) -> int & { return W.pos[i][lane]; };
  auto endp = [&](int i) -> int & { return W.endp[i][lane]; };
  auto tlv = [&](int i) -> int & { return W.tlv[i][lane]; };
  // The last motif edge is real (never an anti-edge).  When it has a root
  // node as its source (target), it lies in that node's out-list (in-list)
  // after the root edge and inside its window, which ends t(e_0) + delta
  // after the root (t(e_0) + gap_0 for a two-edge motif with gaps: edge 1's
  // window may pass delta): a root whose list holds no such entry has no
  // match and is not searched.  side: 0 / 1 in-list of root node 0 / 1,
  // 2 / 3 out-list of root node 0 / 1, -1 none.
  const int last_win = (K == 2 && s.has_temporal) ? s.temporal[0] : s.delta;
  int side = -1;
  if (EVX_CONS_ROOT_DROP) {
    const int wl = s.plan.info[K - 2];
    const int la = plan_a(wl), lb = plan_b(wl);
    side = lb <= 1 ? lb : (la <= 1 ? 2 + la : -1);
  }
  unsigned useout = 0;      // bit j: motif edge j scans an out-list
  int j = 0;                // motif edge being scanned; 0 = between roots
  bool done = false;        // no roots left for this lane
  unsigned long long cnt = 0;

  // open motif edge jj (1 <= jj < K) after the partial match e_0 .. e_{jj-1}
  auto open = [&](int jj) {
    const int w = s.plan.info[jj - 1];
    const int kind = plan_kind(w), a = plan_a(w), b = plan_b(w);
    const int pr = s.prev_real[jj];
    int tl;
    if (s.has_temporal) {
      const int gap = et(pr) + s.temporal[jj - 1];
      tl = (jj >= 2 && et(0) + s.delta < gap) ? et(0) + s.delta : gap;
    } else {
      tl = et(0) + s.delta;
    }
    bool out;
    int lo, hi;
    if (kind == 1) {
      out = true;
    } else if (kind == 0) {
      out = false;
    } else {
      const int4 ra = __ldg(g.node_rng + m(a)), rb = __ldg(g.node_rng + m(b));
      out = !(rb.w - rb.z < ra.y - ra.x);  // the shorter list; ties go to out(a)
    }
    if (out) {
      const int4 r = __ldg(g.node_rng + m(a));
      lo = r.x; hi = r.y;
    } else {
      const int4 r = __ldg(g.node_rng + m(b));
      lo = r.z; hi = r.w;
    }
    lo = first_eid_after(out ? g.out_rec : g.in_rec, lo, hi, eid(pr));
    pos(jj) = lo;
    endp(jj) = hi;
    tlv(jj) = tl;
    useout = out ? (useout | (1u << jj)) : (useout & ~(1u << jj));
    j = jj;
  };

  while (true) {
    // idle lanes claim new roots, one atomic per warp
    const bool idle = (j == 0) && !done;
    const unsigned im = __ballot_sync(0xffffffffu, idle);
    if (im) {
      const int leader = __ffs(im) - 1;
      int base = 0;
      if (lane == leader) {
        const bool stopped = ENUM && !s.exact_total && *(volatile int *)s.stop;
        base = stopped ? s.root_end : atomicAdd(s.cursor, __popc(im));
      }
      base = __shfl_sync(0xffffffffu, base, leader);
      if (idle) {
        const int r = base + __popc(im & ((1u << lane) - 1));
        if (r >= s.root_end) {
          done = true;
        } else {
          const int4 e = __ldg(g.edges + r);
          bool ok = e.x != e.y;
          if (ok && s.node_ok) {
            ok = ((__ldg(s.node_ok + e.x) & 1) != 0) && ((__ldg(s.node_ok + e.y) & 2) != 0);
          }
          if (ok && s.edge_ok) ok = __ldg(s.edge_ok + r) != 0;
          if (ok && side >= 0) {
            const int4 rg = __ldg(g.node_rng + ((side & 1) ? e.y : e.x));
            int st, hi2;
            const int4 *lst;
            if (side < 2) {
              lst = g.in_rec; hi2 = rg.w;
              st = side == 0 ? __ldg(g.cross_in + r) : __ldg(g.inpos + r) + 1;
            } else {
              lst = g.out_rec; hi2 = rg.y;
              st = side == 2 ? e.w + 1 : __ldg(g.cross_out + r);
            }
            ok = st < hi2 && __ldg(&lst[st].z) <= e.z + last_win;
          }
          if (ok) {
            m(0) = e.x;
            m(1) = e.y;
            eid(0) = r;
            et(0) = e.z;
            open(1);
          }
        }
      }
    }
    if (__all_sync(0xffffffffu, done)) break;
    if (j == 0) continue;

    // scan motif edge j
    const int w = s.plan.info[j - 1];
    const int kind = plan_kind(w), a = plan_a(w), b = plan_b(w), nm = plan_nm(w);
    const bool out = (useout >> j) & 1;
    const int4 *__restrict__ recs = out ? g.out_rec : g.in_rec;
    const int want = kind == 2 ? (out ? m(b) : m(a)) : -1;
    const bool anti = (s.anti_mask >> j) & 1;
    const bool last = (j == K - 1);
    const int tl = tlv(j), hi = endp(j);
    int p = pos(j);
    int found = -1, fnode = 0, ft = 0;
    for (; p < hi; p++) {
      const int4 r = __ldg(recs + p);
      if (r.z > tl) { p = hi; break; }
      bool ok;
      if (want >= 0) {
        ok = r.y == want;
      } else {
        ok = true;
#pragma unroll
        for (int q = 0; q < K + 1; q++)
          if (q < nm && m(q) == r.y) ok = false;
        if (ok && s.node_ok) ok = ((__ldg(s.node_ok + r.y) >> nm) & 1) != 0;
      }
      if (ok && s.edge_ok) ok = __ldg(s.edge_ok + r.x) != 0;
      if (!ok) continue;
      if (last) {
        bool pass = true;
        if (s.has_filter) {
          pass = prog_eval(s.filter, [&](int i) -> long long {
                   const int e = i == K - 1 ? r.x : eid(i);
                   return e < 0 ? 0 : __ldg(s.edge_feat + e);
                 }) != 0;
        }
        if (!pass) continue;
        if (ENUM) {
          const unsigned long long slot = atomicAdd(s.count, 1ull);
          if ((long long)slot < s.cap) {
            int *row = s.rows + slot * (unsigned long long)K;
#pragma unroll
            for (int q = 0; q < K - 1; q++) row[q] = eid(q) < 0 ? -1 : __ldg(g.euid + eid(q));
            row[K - 1] = __ldg(g.euid + r.x);
          }
          if ((long long)slot >= s.cap - 1 && !s.exact_total) *(volatile int *)s.stop = 1;
        } else {
          cnt++;
        }
        continue;
      }
      found = r.x;
      fnode = r.y;
      ft = r.z;
      p++;
      break;
    }
    pos(j) = p;
    if (!last && anti && found < 0) {
      eid(j) = -1;  // the edge that must not exist does not: go on
      et(j) = 0;
      open(j + 1);
    } else if (!last && !anti && found >= 0) {
      eid(j) = found;
      et(j) = ft;
      if (kind != 2) m(nm) = fnode;
      open(j + 1);
    } else {
      // window exhausted, or an anti-edge exists: back to the previous real
      // motif edge, whose scan goes on (0: the root is finished)
      j = s.prev_real[j];
    }
  }

  if (!ENUM) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd(s.count, cnt);
  }
}

template <int K>
static int launch_k(const GraphView &g, const ConsSearch &s, bool enumerate, int grid, cudaStream_t st) {
  if (enumerate) cons_search_kernel<K, true><<<grid, kConsBlock, 0, st>>>(g, s);
  else cons_search_kernel<K, false><<<grid, kConsBlock, 0, st>>>(g, s);
  EVX_CUDA(cudaGetLastError());
  return EVX_OK;
}

int launch_constrained(const GraphView &g, const ConsSearch &s, bool enumerate, int grid, cudaStream_t st) {
  switch (s.plan.k) {
    case 2: return launch_k<2>(g, s, enumerate, grid, st);
    case 3: return launch_k<3>(g, s, enumerate, grid, st);
    case 4: return launch_k<4>(g, s, enumerate, grid, st);
    case 5: return launch_k<5>(g, s, enumerate, grid, st);
    case 6: return launch_k<6>(g, s, enumerate, grid, st);
    case 7: return launch_k<7>(g, s, enumerate, grid, st);
    case 8: return launch_k<8>(g, s, enumerate, grid, st);
    default: return fail(EVX_ERR_INVALID, "motif size out of range");
  }
}

template <int K>
static int occ_k(bool enumerate, int *bps) {
  cudaError_t e = enumerate
      ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, cons_search_kernel<K, true>, kConsBlock, 0)
      : cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, cons_search_kernel<K, false>, kConsBlock, 0);
  if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  return EVX_OK;
}

int cons_occupancy(int k, bool enumerate, int *bps) {
  switch (k) {
    case 2: return occ_k<2>(enumerate, bps);
    case 3: return occ_k<3>(enumerate, bps);
    case 4: return occ_k<4>(enumerate, bps);
    case 5: return occ_k<5>(enumerate, bps);
    case 6: return occ_k<6>(enumerate, bps);
    case 7: return occ_k<7>(enumerate, bps);
    case 8: return occ_k<8>(enumerate, bps);
    default: return fail(EVX_ERR_INVALID, "motif size out of range");
  }
}

int cons_block() { return kConsBlock; }

}  // namespace evx
