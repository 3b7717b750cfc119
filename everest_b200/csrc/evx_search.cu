// Per-motif backtracking search for temporal motifs on sm_100a.
//
// Semantics (bit-exact with the reference's generated kernel,
// system/templates/dispatch/top.snp and system/templates/common/*.snp):
// a match is a tuple of edge ids e_0 < e_1 < ... < e_{k-1} with
// u(e_0) != v(e_0), t(e_j) <= t(e_0) + delta, and an injective map of motif
// nodes to graph nodes.  Motif edge j >= 1 is searched in the out-list of the
// image of its source when its target is new, the in-list of the image of its
// target when its source is new, and the shorter of the two when both are
// mapped (system/templates/common/resolveMi.snp:1-28).
//
// B200 design (not a translation of the reference's per-lane register DFS):
//  * adjacency entries are packed 16-byte records {eid, other, t, pos}; one
//    ld.global.nc.v4 replaces the reference's two dependent gathers
//    (i_S[beg] then the 12-byte AoS Eg[idx],
//    system/templates/common/nextMatchInTask.snp:3-4); per-node ranges are
//    one int4 {out_beg, out_end, in_beg, in_end};
//  * each lane runs its DFS as a state machine (ROOT -> OPEN -> BSEARCH ->
//    SCAN, with pops in between) in which every iteration issues exactly one
//    round of independent loads per lane and then does only ALU work, so the
//    lanes of a warp overlap their memory latency even while they are in
//    different phases (the reference executes a list opening's binary search
//    inline, serialising the warp on it, system/templates/funcs/reduceEarlyIdx.snp);
//  * a list opening finds its start in O(1) when the list is the previous
//    edge's own out/in list (the record carries the edge's position in its
//    other list), otherwise by a binary search advanced one probe per iteration;
//  * the last level reads two records per iteration;
//  * lanes are refilled with new roots one by one from a per-warp pool as
//    soon as they finish (the reference refills a warp only when all 32
//    lanes are done, system/templates/warpCentric/tidEnd.snp);
//  * when the global root cursor is exhausted, idle lanes split the
//    shallowest, widest remaining candidate range of one donor lane into
//    equal contiguous parts (warp shuffle of the donor state, exact
//    partition), in place of the reference's one-candidate-per-thief split
//    (system/templates/warpBalancing/top.snp) and its host-driven
//    dump/expand rounds (system/templates/tailExpan/Expanding.snp);
//  * enumeration slots are reserved with one warp-aggregated atomicAdd per
//    iteration (the reference issues one atomicAdd per match,
//    system/tmine/KernelGen.py:505-524).
#include "evx_internal.cuh"

namespace evx {
namespace {

constexpr unsigned kFull = 0xffffffffu;

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

// First position in [lo, hi) whose edge id is greater than prev.
__device__ __forceinline__ int first_eid_after(const int4 *lst, int lo, int hi, int prev) {
  if (lo >= hi) return hi;
  if (ld_eid(lst + hi - 1) <= prev) return hi;
  if (ld_eid(lst + lo) > prev) return lo;
  int a = lo + 1, b = hi - 1;  // eid(b) > prev, eid(lo) <= prev
  while (a < b) {
    int mid = (a + b) >> 1;
    if (ld_eid(lst + mid) > prev) b = mid; else a = mid + 1;
  }
  return a;
}

// First position in [lo, hi) whose timestamp is greater than tv.
__device__ __forceinline__ int first_t_after(const int4 *lst, int lo, int hi, int tv) {
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (ld_t(lst + mid) > tv) hi = mid; else lo = mid + 1;
  }
  return lo;
}

template <int K, bool ENUM>
__global__ void __launch_bounds__(256)
search_kernel(const GraphView g, const MotifPlan plan, const SearchArgs args) {
  constexpr int L = K - 1;                 // search levels (motif edges 1..k-1)
  constexpr int N = K + 1;                 // motif nodes <= k + 1
  constexpr int S = (L > 1) ? (L - 1) : 1; // saved ranges for levels 0..L-2
  constexpr int KE = ENUM ? K : 1;
  constexpr bool WIDE = !ENUM;             // two records per last-level step
  enum : int { M_IDLE = 0, M_ROOT = 1, M_OPEN = 2, M_BS = 3, M_SCAN = 4 };

  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  const int strict = args.strict_ts;

  int info[L];
#pragma unroll
  for (int l = 0; l < L; l++) info[l] = plan.info[l];

  int m[N];
#pragma unroll
  for (int q = 0; q < N; q++) m[q] = -1;
  int e[KE];
#pragma unroll
  for (int q = 0; q < KE; q++) e[q] = 0;
  int sp[S], se[S];
#pragma unroll
  for (int q = 0; q < S; q++) { sp[q] = 0; se[q] = 0; }

  int mode = M_IDLE, level = -1;
  int pos = 0, end = 0, bhi = 0;  // SCAN: [pos, end); BSEARCH: window [pos, bhi)
  int tl = 0, want = -1, base = 0, nmc = 0;
  bool out = true;
  unsigned iomask = 0;
  int key = 0, sc0 = -1, sc1 = -1, n0 = 0, n1 = -1;  // pending OPEN (n0 = root id in ROOT)
  unsigned long long cnt = 0;

  int pool_next = 0, pool_end = 0;
  bool exhausted = false;
  unsigned iter = 0;

  // (Re)derive list / target of level l from the plan, the node images and
  // the saved list choice.
  auto restore = [&](int l) {
    const int w = sel(info, l);
    const int kind = plan_kind(w);
    nmc = plan_nm(w);
    out = (iomask >> l) & 1u;
    const int ia = sel(m, plan_a(w)), ib = sel(m, plan_b(w));
    if (kind == 2) { base = out ? ia : ib; want = out ? ib : ia; }
    else { base = (kind == 1) ? ia : ib; want = -1; }
  };

  // Queue the opening of level l's list after matching edge peid
  // (t pt, endpoints psrc->pdst, positions pop in out_rec / pip in in_rec).
  auto prepare_open = [&](int l, int peid, int pt, int psrc, int pdst, int pop, int pip) {
    const int w = sel(info, l);
    const int kind = plan_kind(w);
    const int ia = sel(m, plan_a(w)), ib = sel(m, plan_b(w));
    key = strict ? pt : peid;
    if (kind == 2) {
      n0 = ib; n1 = ia;
      sc0 = (pdst == ib) ? pip + 1 : -1;
      sc1 = (psrc == ia) ? pop + 1 : -1;
    } else if (kind == 1) {
      n0 = ia; n1 = -1;
      sc0 = -1;
      sc1 = (psrc == ia) ? pop + 1 : -1;
    } else {
      n0 = ib; n1 = -1;
      sc0 = (pdst == ib) ? pip + 1 : -1;
      sc1 = -1;
    }
    mode = M_OPEN;
  };

  auto structural_ok = [&](int node) -> bool {
    if (want >= 0) return node == want;
    bool ok = true;
#pragma unroll
    for (int q = 0; q < N; q++) ok = ok && !(q < nmc && m[q] == node);
    return ok;
  };

  while (true) {
    ++iter;
    // ---------------------------------------------------- root refill ----
    const unsigned idle = __ballot_sync(kFull, mode == M_IDLE);
    if (idle && !exhausted) {
      const int nidle = __popc(idle);
      const int rank = __popc(idle & lt_mask);
      const int avail = pool_end - pool_next;
      int nb = 0, nbe = 0;
      bool stopped = false;
      if (ENUM) {
        int sflag = 0;
        if (lane == 0) sflag = *(volatile int *)args.stop;
        stopped = __shfl_sync(kFull, sflag, 0) != 0;
      }
      if (stopped) {
        exhausted = true;
      } else {
        if (avail < nidle) {
          int got = 0;
          if (lane == 0) got = atomicAdd(args.cursor, args.roots_per_fetch);
          got = __shfl_sync(kFull, got, 0);
          nb = min(got, args.root_end);
          nbe = min(got + args.roots_per_fetch, args.root_end);
        }
        if (mode == M_IDLE) {
          int r = -1;
          if (rank < avail) r = pool_next + rank;
          else if (nb + (rank - avail) < nbe) r = nb + (rank - avail);
          if (r >= 0) { n0 = r; mode = M_ROOT; }
        }
        if (avail >= nidle) {
          pool_next += nidle;
        } else {
          pool_next = min(nb + (nidle - avail), nbe);
          pool_end = nbe;
          if (nb >= nbe) exhausted = true;
        }
      }
    }

    // ----------------------------------------- issue this step's loads ----
    int4 r0 = make_int4(0, 0, 0, 0), r1 = make_int4(0, 0, 0, 0);
    int x0 = 0;
    bool two = false;
    {
      const int4 *lst = out ? g.out_rec : g.in_rec;
      if (mode == M_SCAN) {
        r0 = __ldg(lst + pos);
        two = WIDE && (level == L - 1) && (pos + 1 < end);
        if (two) r1 = __ldg(lst + pos + 1);
      } else if (mode == M_BS) {
        const int mid = (pos + bhi) >> 1;
        x0 = strict ? ld_t(lst + mid) : ld_eid(lst + mid);
      } else if (mode == M_OPEN) {
        r0 = __ldg(g.node_rng + n0);
        if (n1 >= 0) r1 = __ldg(g.node_rng + n1);
      } else if (mode == M_ROOT) {
        r0 = __ldg(g.edges + n0);
        x0 = __ldg(g.inpos + n0);
      }
    }

    // ------------------------------------------------ process the step ----
    bool emit = false;
    int last_eid = 0;
    if (mode == M_SCAN) {
      ++pos;
      if (r0.z > tl) {
        pos = end;  // rest of the list is outside the window
      } else if (structural_ok(r0.y)) {
        if (level == L - 1) {
          ++cnt;
          if (ENUM) { emit = true; last_eid = r0.x; }
        } else {
          put(sp, level, pos);
          put(se, level, end);
          if (want < 0) put(m, nmc, r0.y);
          if (ENUM) put(e, level + 1, r0.x);
          const int psrc = out ? base : r0.y;
          const int pdst = out ? r0.y : base;
          const int pop = out ? pos - 1 : r0.w;
          const int pip = out ? r0.w : pos - 1;
          ++level;
          prepare_open(level, r0.x, r0.z, psrc, pdst, pop, pip);
        }
      }
      if (two && pos < end) {  // second record of a last-level step
        ++pos;
        if (r1.z > tl) pos = end;
        else if (structural_ok(r1.y)) ++cnt;
      }
    } else if (mode == M_BS) {
      const int mid = (pos + bhi) >> 1;
      if (x0 > key) bhi = mid; else pos = mid + 1;
      if (pos >= bhi) mode = M_SCAN;  // pos = first record after the previous edge
    } else if (mode == M_OPEN) {
      const int w = sel(info, level);
      const int kind = plan_kind(w);
      nmc = plan_nm(w);
      const int ia = sel(m, plan_a(w)), ib = sel(m, plan_b(w));
      int lo, hi, sc;
      if (kind == 2) {
        if (r0.w - r0.z < r1.y - r1.x) { out = false; base = ib; want = ia; lo = r0.z; hi = r0.w; sc = sc0; }
        else { out = true; base = ia; want = ib; lo = r1.x; hi = r1.y; sc = sc1; }
      } else if (kind == 1) {
        out = true; base = ia; want = -1; lo = r0.x; hi = r0.y; sc = sc1;
      } else {
        out = false; base = ib; want = -1; lo = r0.z; hi = r0.w; sc = sc0;
      }
      iomask = (iomask & ~(1u << level)) | ((unsigned)out << level);
      end = hi;
      if (!strict && sc >= 0) { pos = sc; mode = M_SCAN; }
      else if (lo >= hi) { pos = hi; mode = M_SCAN; }
      else { pos = lo; bhi = hi; mode = M_BS; }
    } else if (mode == M_ROOT) {
      if (r0.x == r0.y) {  // self-loops are not roots
        mode = M_IDLE;
      } else {
        m[0] = r0.x;
        m[1] = r0.y;
        tl = r0.z + args.delta;
        if (ENUM) e[0] = n0;
        level = 0;
        prepare_open(0, n0, r0.z, r0.x, r0.y, r0.w, x0);
      }
    }
    // exhausted ranges: pop to the deepest level with work left
    while (mode == M_SCAN && pos >= end) {
      if (level == 0) { mode = M_IDLE; level = -1; }
      else { --level; pos = sel(sp, level); end = sel(se, level); restore(level); }
    }

    // ------------------------------------------- enumeration output ----
    if (ENUM) {
      const unsigned em = __ballot_sync(kFull, emit);
      if (em) {
        const int leader = __ffs(em) - 1;
        unsigned long long b0 = 0;
        if (lane == leader) b0 = atomicAdd(args.count, (unsigned long long)__popc(em));
        b0 = __shfl_sync(kFull, b0, leader);
        if (emit) {
          const unsigned long long slot = b0 + (unsigned long long)__popc(em & lt_mask);
          if (slot < (unsigned long long)args.cap) {
            int *row = args.rows + slot * K;
#pragma unroll
            for (int q = 0; q < K - 1; q++) row[q] = __ldg(g.euid + e[q < KE ? q : 0]);
            row[K - 1] = __ldg(g.euid + last_eid);
          }
          if (!args.exact_total && slot + 1 >= (unsigned long long)args.cap)
            atomicExch(args.stop, 1);
        }
      }
    }

    // ---------------------------------------- tail: finish or steal ----
    if (exhausted) {
      const unsigned idle2 = __ballot_sync(kFull, mode == M_IDLE);
      if (idle2 == kFull) break;
      if (idle2 && args.steal_interval && (iter & (unsigned)(args.steal_interval - 1)) == 0) {
        // shallowest level with a splittable remaining range, then widest
        int sl = -1, sw = 0;
        if (mode != M_IDLE) {
#pragma unroll
          for (int l = 0; l < S; l++) {
            if (sl < 0 && l < level) {
              const int w = se[l] - sp[l];
              if (w >= args.min_split) { sl = l; sw = w; }
            }
          }
          if (sl < 0 && mode == M_SCAN && end - pos >= args.min_split) { sl = level; sw = end - pos; }
        }
        const unsigned skey = sl < 0 ? 0u : (((unsigned)(L - sl) << 24) | (unsigned)min(sw, 0xFFFFFF));
        const unsigned kmax = __reduce_max_sync(kFull, skey);
        if (kmax) {
          const int donor = __ffs(__ballot_sync(kFull, skey == kmax)) - 1;
          const int split_l = L - (int)(kmax >> 24);
          int p0 = 0, p1 = 0;
          if (lane == donor) {
            const bool cur = (split_l == level);
            p0 = cur ? pos : sel(sp, split_l);
            p1 = cur ? end : sel(se, split_l);
            const bool o = (iomask >> split_l) & 1u;
            p1 = first_t_after(o ? g.out_rec : g.in_rec, p0, p1, tl);  // window end
            if (cur) end = p1; else put(se, split_l, p1);
          }
          p0 = __shfl_sync(kFull, p0, donor);
          p1 = __shfl_sync(kFull, p1, donor);
          const int w = p1 - p0;
          const int nthief = min(__popc(idle2), w - 1);
          if (nthief > 0) {
            const int parts = nthief + 1;
            const int rank = __popc(idle2 & lt_mask);
            const bool thief = (mode == M_IDLE) && rank < nthief;
#pragma unroll
            for (int q = 0; q < N; q++) {
              const int x = __shfl_sync(kFull, m[q], donor);
              if (thief) m[q] = x;
            }
            if (ENUM) {
#pragma unroll
              for (int q = 0; q < KE; q++) {
                const int x = __shfl_sync(kFull, e[q], donor);
                if (thief) e[q] = x;
              }
            }
            const int dtl = __shfl_sync(kFull, tl, donor);
            const unsigned dio = __shfl_sync(kFull, iomask, donor);
            if (thief) {
              tl = dtl;
              iomask = dio;
              level = split_l;
              mode = M_SCAN;
              pos = p0 + (int)((long long)w * (rank + 1) / parts);
              end = p0 + (int)((long long)w * (rank + 2) / parts);
#pragma unroll
              for (int q = 0; q < S; q++) { sp[q] = 0; se[q] = 0; }
              restore(split_l);
            }
            if (lane == donor) {
              const int ne = p0 + (int)((long long)w / parts);
              if (split_l == level) end = ne; else put(se, split_l, ne);
            }
          } else if (lane == donor) {
            // nothing to split after trimming: drop an exhausted range
            while (mode == M_SCAN && pos >= end) {
              if (level == 0) { mode = M_IDLE; level = -1; }
              else { --level; pos = sel(sp, level); end = sel(se, level); restore(level); }
            }
          }
        }
      }
    }
  }

  if (!ENUM) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(kFull, cnt, o);
    if (lane == 0 && cnt) atomicAdd(args.count, cnt);
  }
}

template <int K, bool ENUM>
int launch_k(const GraphView &g, const MotifPlan &plan, const SearchArgs &args, int grid,
             int block, cudaStream_t s) {
  search_kernel<K, ENUM><<<grid, block, 0, s>>>(g, plan, args);
  return 0;
}

template <int K, bool ENUM>
int occ_k(int block, int *bps) {
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, search_kernel<K, ENUM>, block, 0);
  return e == cudaSuccess ? 0 : cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
}

}  // namespace

#define EVX_K_DISPATCH(FN, ...)                                        \
  switch (k) {                                                         \
    case 2: return enumerate ? FN<2, true>(__VA_ARGS__) : FN<2, false>(__VA_ARGS__); \
    case 3: return enumerate ? FN<3, true>(__VA_ARGS__) : FN<3, false>(__VA_ARGS__); \
    case 4: return enumerate ? FN<4, true>(__VA_ARGS__) : FN<4, false>(__VA_ARGS__); \
    case 5: return enumerate ? FN<5, true>(__VA_ARGS__) : FN<5, false>(__VA_ARGS__); \
    case 6: return enumerate ? FN<6, true>(__VA_ARGS__) : FN<6, false>(__VA_ARGS__); \
    case 7: return enumerate ? FN<7, true>(__VA_ARGS__) : FN<7, false>(__VA_ARGS__); \
    case 8: return enumerate ? FN<8, true>(__VA_ARGS__) : FN<8, false>(__VA_ARGS__); \
    default: return fail(EVX_ERR_INVALID, "motif edge count out of range");          \
  }

int launch_search(const GraphView &g, const MotifPlan &plan, const SearchArgs &args, int grid,
                  int block, cudaStream_t stream) {
  const int k = plan.k;
  const bool enumerate = args.enumerate != 0;
  EVX_K_DISPATCH(launch_k, g, plan, args, grid, block, stream)
}

int search_occupancy(int k, bool enumerate, int block, int *blocks_per_sm) {
  EVX_K_DISPATCH(occ_k, block, blocks_per_sm)
}

}  // namespace evx
