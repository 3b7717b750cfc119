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
//    system/templates/common/nextMatchInTask.snp:3-4);
//  * every list opening finds its start in O(1) when the list is the
//    previous edge's own out/in list (the record carries the edge's position
//    in its other list), otherwise by a binary search over the records
//    (system/templates/funcs/reduceEarlyIdx.snp);
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

  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;

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

  int level = -1;  // -1: lane idle (needs a root)
  int pos = 0, end = 0, tl = 0;
  int want = -1, base = 0, nmc = 0;
  bool out = true;
  unsigned iomask = 0;
  unsigned long long cnt = 0;

  int pool_next = 0, pool_end = 0;
  bool exhausted = false;
  unsigned iter = 0;
  const int strict = args.strict_ts;

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

  // Open the candidate list of level l given the previous matched edge.
  auto open = [&](int l, int peid, int pt, int psrc, int pdst, int pop, int pip) {
    const int w = sel(info, l);
    const int kind = plan_kind(w);
    nmc = plan_nm(w);
    const int ia = sel(m, plan_a(w)), ib = sel(m, plan_b(w));
    int lo, hi;
    if (kind == 2) {
      const int i0 = __ldg(g.in_off + ib), i1 = __ldg(g.in_off + ib + 1);
      const int o0 = __ldg(g.out_off + ia), o1 = __ldg(g.out_off + ia + 1);
      if (i1 - i0 < o1 - o0) { out = false; base = ib; want = ia; lo = i0; hi = i1; }
      else { out = true; base = ia; want = ib; lo = o0; hi = o1; }
    } else {
      out = (kind == 1);
      base = out ? ia : ib;
      want = -1;
      const int *off = out ? g.out_off : g.in_off;
      lo = __ldg(off + base);
      hi = __ldg(off + base + 1);
    }
    iomask = (iomask & ~(1u << l)) | ((unsigned)out << l);
    const int4 *lst = out ? g.out_rec : g.in_rec;
    if (strict) {
      lo = first_t_after(lst, lo, hi, pt);
    } else if (out && base == psrc) {
      lo = pop + 1;
    } else if (!out && base == pdst) {
      lo = pip + 1;
    } else {
      lo = first_eid_after(lst, lo, hi, peid);
    }
    pos = lo;
    end = hi;
  };

  while (true) {
    ++iter;
    // ---------------------------------------------------- root refill ----
    unsigned idle = __ballot_sync(kFull, level < 0);
    if (idle && !exhausted) {
      const int nidle = __popc(idle);
      const int rank = __popc(idle & lt_mask);
      const int avail = pool_end - pool_next;
      int nb = 0, nbe = 0;
      bool stopped = false;
      if (ENUM) {
        int s = 0;
        if (lane == 0) s = *(volatile int *)args.stop;
        stopped = __shfl_sync(kFull, s, 0) != 0;
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
        int r = -1;
        if (level < 0) {
          if (rank < avail) r = pool_next + rank;
          else if (nb + (rank - avail) < nbe) r = nb + (rank - avail);
        }
        if (avail >= nidle) {
          pool_next += nidle;
        } else {
          pool_next = min(nb + (nidle - avail), nbe);
          pool_end = nbe;
          if (nb >= nbe) exhausted = true;
        }
        if (r >= 0) {
          const int4 ed = __ldg(g.edges + r);
          if (ed.x != ed.y) {  // self-loops are not roots
            m[0] = ed.x;
            m[1] = ed.y;
            tl = ed.z + args.delta;
            if (ENUM) e[0] = r;
            level = 0;
            const int2 rp = __ldg(g.rootpos + r);
            open(0, r, ed.z, ed.x, ed.y, rp.x, rp.y);
          }
        }
      }
    }

    // -------------------------------------------------- one DFS step ----
    bool emit = false;
    int last_eid = 0;
    if (level >= 0) {
      if (pos < end) {
        const int4 *lst = out ? g.out_rec : g.in_rec;
        const int4 rc = __ldg(lst + pos);
        ++pos;
        if (rc.z > tl) {
          end = pos;  // rest of the list is outside the window
        } else {
          bool ok;
          if (want >= 0) {
            ok = (rc.y == want);
          } else {
            ok = true;
#pragma unroll
            for (int q = 0; q < N; q++) ok = ok && !(q < nmc && m[q] == rc.y);
          }
          if (ok) {
            if (level == L - 1) {
              ++cnt;
              if (ENUM) { emit = true; last_eid = rc.x; }
            } else {
              put(sp, level, pos);
              put(se, level, end);
              if (want < 0) put(m, nmc, rc.y);
              if (ENUM) put(e, level + 1, rc.x);
              const int psrc = out ? base : rc.y;
              const int pdst = out ? rc.y : base;
              const int pop = out ? pos - 1 : rc.w;
              const int pip = out ? rc.w : pos - 1;
              ++level;
              open(level, rc.x, rc.z, psrc, pdst, pop, pip);
            }
          }
        }
      } else if (level == 0) {
        level = -1;  // root finished
      } else {
        --level;
        pos = sel(sp, level);
        end = sel(se, level);
        restore(level);
      }
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
            for (int q = 0; q < K - 1; q++) row[q] = __ldg(&g.edges[e[q < KE ? q : 0]].w);
            row[K - 1] = __ldg(&g.edges[last_eid].w);
          }
          if (!args.exact_total && slot + 1 >= (unsigned long long)args.cap)
            atomicExch(args.stop, 1);
        }
      }
    }

    // ---------------------------------------- tail: finish or steal ----
    if (exhausted) {
      const unsigned idle2 = __ballot_sync(kFull, level < 0);
      if (idle2 == kFull) break;
      if (idle2 && args.steal_interval && (iter & (unsigned)(args.steal_interval - 1)) == 0) {
        // shallowest level with a splittable remaining range, then widest
        int sl = -1, sw = 0;
        if (level >= 0) {
#pragma unroll
          for (int l = 0; l < S; l++) {
            if (sl < 0 && l < level) {
              const int w = se[l] - sp[l];
              if (w >= args.min_split) { sl = l; sw = w; }
            }
          }
          if (sl < 0 && end - pos >= args.min_split) { sl = level; sw = end - pos; }
        }
        const unsigned key = sl < 0 ? 0u : (((unsigned)(L - sl) << 24) | (unsigned)min(sw, 0xFFFFFF));
        const unsigned kmax = __reduce_max_sync(kFull, key);
        if (kmax) {
          const int donor = __ffs(__ballot_sync(kFull, key == kmax)) - 1;
          const int split_l = L - (int)(kmax >> 24);
          int p0 = 0, p1 = 0;
          if (lane == donor) {
            p0 = (split_l == level) ? pos : sel(sp, split_l);
            p1 = (split_l == level) ? end : sel(se, split_l);
            const bool o = (iomask >> split_l) & 1u;
            p1 = first_t_after(o ? g.out_rec : g.in_rec, p0, p1, tl);  // window end
            if (split_l == level) end = p1; else put(se, split_l, p1);
          }
          p0 = __shfl_sync(kFull, p0, donor);
          p1 = __shfl_sync(kFull, p1, donor);
          const int w = p1 - p0;
          const int nthief = min(__popc(idle2), w - 1);
          if (nthief > 0) {
            const int parts = nthief + 1;
            const int rank = __popc(idle2 & lt_mask);
            const bool thief = (level < 0) && rank < nthief;
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
