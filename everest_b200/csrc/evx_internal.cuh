// Internal types shared by the device graph, search kernels and C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/everest_b200.h"

namespace evx {

// Device layout of one graph (all int32; E < 2^31, V < 2^31).
//   edges[e]    = {u, v, t, position of e in out_rec}     root fetch
//   inpos[e]    = position of e in in_rec
//   euid[e]     = original line id of e                    enumeration rows
//   out_rec[p]  = {eid, v, t, position of eid in in_rec (low bits; see kPosMask)}   grouped by u, ascending eid
//   in_rec[p]   = {eid, u, t, position of eid in out_rec}  grouped by v, ascending eid
//   node_rng[x] = {out_beg, out_end, in_beg, in_end}       positions in out_rec / in_rec
//   pair_rec[i] = {eid, t} grouped by static edge (u, v), ascending eid
//   pair_tab[h] = {v, u, start, len}: open-addressing table (u, v) -> run in pair_rec
//                 (the first 8 bytes hold the 64-bit key; all ones = empty)
// Positions are absolute indices into out_rec / in_rec.
struct GraphView {
  const int4 *edges;
  const int *inpos;
  const int *euid;
  const int4 *out_rec;
  const int4 *in_rec;
  const int4 *node_rng;
  const int4 *pair_tab;
  const int2 *pair_rec;
  const int2 *pair_loc;       // [e] = {position of e in pair_rec, end of its run}
  const int *cross_out;       // [e] = first position of out(v) holding an edge after e = (u, v)
  const int *cross_in;        // [e] = first position of in(u) holding an edge after e = (u, v)
  const int2 *rev_loc;        // [e] = {first position after e in the run of the reverse
                              //        pair (v, u), end of that run}; {0, 0} when no v->u edge
  const int2 *pair_dir;       // [r] = {v, start} of run r, sorted by (u, v); [P] = sentinel
  const int *dir_off;         // [u] = first run of source u (V + 1 entries)
  const unsigned long long *sig_out;  // [u] = OR of 1 << sig_bit(v) over u's out-neighbours v
  const unsigned long long *sig_in;   // [v] = OR of 1 << sig_bit(u) over v's in-neighbours u
  unsigned long long pair_mask;
  int pair_max_probe;
  int num_edges;
  int num_vertices;
};

__host__ __device__ inline unsigned long long pair_key(int u, int v) {
  return ((unsigned long long)(unsigned)u << 32) | (unsigned long long)(unsigned)v;
}

// 64-bit finalizer (splitmix64 constants) used as the pair-table hash.
__host__ __device__ inline unsigned long long pair_hash(unsigned long long x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return x;
}

// The fourth word of an out_rec / in_rec record: the edge's position in its
// other list in the low 30 bits; the top bit is set when the edge's pair run
// (same endpoints, same direction) has a later entry, and bit 30 when its
// reverse pair's run has an entry after it (graphs hold fewer than 2^30
// edges, alloc_graph in evx_capi.cu, so positions fit in 30 bits).
constexpr int kPosMask = 0x3fffffff;
constexpr int kRevLater = 0x40000000;

// Bit of a node in the 64-bit neighbour signatures (Fibonacci hashing; a
// different hash from the pair table's).
__host__ __device__ inline int sig_bit(int x) {
  return (int)(((unsigned long long)(unsigned)x * 0x9E3779B97F4A7C15ull) >> 58);
}

// False only when no u -> v edge exists: both signatures are small enough to
// stay in L2, so most absent pairs are rejected without touching the pair
// table.
__device__ __forceinline__ bool pair_maybe(const GraphView &g, int u, int v) {
  const unsigned long long so = __ldg(g.sig_out + u), si = __ldg(g.sig_in + v);
  return ((so >> sig_bit(v)) & (si >> sig_bit(u)) & 1ull) != 0;
}

// (start, len) of the run of u->v edges in pair_rec; len 0 when absent.  The
// probe sequence stops at the longest one the table build used.
__device__ __forceinline__ int2 pair_find(const GraphView &g, int u, int v) {
  const unsigned long long key = pair_key(u, v);
  unsigned long long h = pair_hash(key) & g.pair_mask;
  for (int i = 0; i < g.pair_max_probe; i++) {
    const int4 s = __ldg(g.pair_tab + h);
    const unsigned long long k = ((unsigned long long)(unsigned)s.y << 32) | (unsigned)s.x;
    if (k == key) return make_int2(s.z, s.w);
    if (k == ~0ull) break;
    h = (h + 1) & g.pair_mask;
  }
  return make_int2(0, 0);
}

// Per-level search plan.  Level l (0-based) matches motif edge j = l + 1.
//   kind 0: new source -> scan in-list of image(b)
//   kind 1: new target -> scan out-list of image(a)
//   kind 2: both mapped -> scan the shorter of in(image(b)) / out(image(a))
// nm = nodes mapped before edge j (= index of the new node for kinds 0/1).
// Packed as kind | a << 4 | b << 8 | nm << 12.
struct MotifPlan {
  int k;          // motif edges
  int n;          // motif nodes
  int info[EVX_MAX_MOTIF_EDGES];
};

__host__ __device__ inline int plan_kind(int w) { return w & 3; }
__host__ __device__ inline int plan_a(int w) { return (w >> 4) & 15; }
__host__ __device__ inline int plan_b(int w) { return (w >> 8) & 15; }
__host__ __device__ inline int plan_nm(int w) { return (w >> 12) & 15; }

// One query of a search launch (a table of these drives the batched kernel).
constexpr int kQStrict = 1;      // t(e_j) > t(e_{j-1}) as well
constexpr int kQInlineLast = 2;  // closing last edge counted on the pair index
constexpr int kQSamePair = 4;    // last edge repeats the previous edge's endpoints
constexpr int kQPairDir = 8;     // last edge's pair found through the per-node pair directory
constexpr int kQPairHash = 16;   // last edge's pair found through the pair hash table
constexpr int kQNoPrune = 32;    // no closing-endpoint check before a task's scan
constexpr int kQRevPair = 64;    // last edge reverses the previous edge's endpoints
constexpr int kQNewArith = 128;  // a new-node last edge's long windows counted by range arithmetic
constexpr int kQPairScan = 256;  // a scanned edge between two mapped nodes walks its pair run
constexpr int kQNoBound = 512;   // no per-root window bound from the last edge's list
struct QueryDesc {
  MotifPlan plan;
  int root_beg, root_end;  // root edge ids [beg, end)
  int delta;
  int flags;               // kQ* bits
  int steal_interval;      // steps between rebalances (power of two), 0 = never
  int min_split;           // smallest range worth splitting
  int tile_beg;            // first work-queue tile of this query
  int pad;
};

// Enumeration outputs (single-query enumerate launches only).
struct EnumArgs {
  int *rows;                  // [cap * k] original line ids
  long long cap;
  int exact_total;            // keep counting past the cap
  int *stop;                  // set when the cap is reached: stop claiming roots
  unsigned long long *count;  // slot counter (= reported count)
};

// A search launch: nq queries sharing one work queue of root tiles.
// Node / edge predicates and temporal gaps of a constrained single query run
// by the warp-synchronous search (no anti-edge, no filter; those take the
// per-lane constrained kernel).  All null / zero for a plain query.
struct ConsArgs {
  const unsigned short *node_ok;  // [V] bit a: the node may be motif node a (null: all)
  const unsigned char *edge_ok;   // [E] edge predicate (null: all)
  int has_gap;                    // motif edge j (j >= 1) ends its window at
  int gap[EVX_MAX_MOTIF_EDGES];   // [j-1]: t(e_{j-1}) + gap, not after t(e_0) + delta (j >= 2)
};

struct LaunchArgs {
  const QueryDesc *table;     // device table (nq > 1); ignored when nq == 1
  int nq;
  int total_tiles;
  int tile_roots;             // roots per tile (multiple of 32)
  int *cursor;                // next unclaimed tile
  unsigned long long *counts; // [nq] per-query counts
  unsigned long long limit;   // work limit per query (0 = none): a query whose
                              // meter passes it is stopped early
  unsigned long long *meter;  // [nq] matches + queued partial matches per query
                              // (maintained only when limit > 0)
  ConsArgs cons;              // single constrained query (the CS kernels); zero otherwise
};

// Search job arguments (one query).
struct SearchArgs {
  int root_beg, root_end;     // root edge ids [beg, end)
  int delta;
  int strict_ts;
  int roots_per_fetch;        // roots claimed per warp refill (multiple of 1)
  int steal_interval;         // iterations between steal checks (power of 2), 0 = off
  int min_split;              // smallest range width worth splitting
  int enumerate;              // 1: write rows
  int tail_flags;             // kQInlineLast / kQSamePair: how the last edge is counted
  int exact_total;            // enumerate: keep counting past the cap
  long long cap;              // enumeration rows capacity
  int *rows;                  // [cap * k] original line ids
  unsigned long long *count;  // [1] result / enumeration slot counter
  int *cursor;                // [1] next unclaimed root id
  int *stop;                  // [1] set when the enumeration cap is reached
  unsigned long long limit;   // work limit (0 = none), count mode only
  unsigned long long *meter;  // [1] matches + queued partial matches (limit > 0)
  ConsArgs cons;              // node / edge predicates and temporal gaps (zero: none)
};

// Host-side graph object.
struct DeviceGraph {
  int device = 0;
  cudaStream_t stream = nullptr;  // stream its memory was allocated on
  int64_t num_edges = 0, num_vertices = 0;
  int max_t = 0, min_t = 0;
  int4 *edges = nullptr;
  int *inpos = nullptr;
  int *euid = nullptr;
  int4 *out_rec = nullptr;
  int4 *in_rec = nullptr;
  int4 *node_rng = nullptr;
  int4 *pair_tab = nullptr;
  int2 *pair_rec = nullptr;
  int2 *pair_loc = nullptr;
  int2 *rev_loc = nullptr;
  int *cross_out = nullptr, *cross_in = nullptr;
  int2 *pair_dir = nullptr;
  int *dir_off = nullptr;
  unsigned long long *sig_out = nullptr, *sig_in = nullptr;
  int *node_feat = nullptr, *edge_feat = nullptr;  // constraint features (optional)
  unsigned long long pair_mask = 0;
  int pair_max_probe = 0;
  int64_t bytes = 0;
  GraphView view() const {
    GraphView g;
    g.edges = edges; g.inpos = inpos; g.euid = euid; g.out_rec = out_rec; g.in_rec = in_rec;
    g.node_rng = node_rng;
    g.pair_tab = pair_tab; g.pair_rec = pair_rec; g.pair_loc = pair_loc; g.pair_mask = pair_mask;
    g.rev_loc = rev_loc; g.cross_out = cross_out; g.cross_in = cross_in;
    g.pair_dir = pair_dir; g.dir_off = dir_off; g.sig_out = sig_out; g.sig_in = sig_in;
    g.pair_max_probe = pair_max_probe;
    g.num_edges = (int)num_edges; g.num_vertices = (int)num_vertices;
    return g;
  }
};

// Decode relabeled motif edges into the per-level plan (evx_capi.cu).
int build_plan(int k, const int *mu, const int *mv, MotifPlan *plan);
// How a count query counts its last edge (kQInlineLast, kQSamePair or 0).
int tail_mode(const MotifPlan &plan, unsigned flags, bool enumerate);

// Stream-ordered device allocations from a library-owned pool per device
// that keeps freed memory mapped (graph re-uploads and pair-index scratch
// reuse it instead of paying for fresh cudaMalloc / cudaFree each time).
cudaError_t dev_alloc(void **p, size_t bytes, int device, cudaStream_t s);
void dev_free(void *p, cudaStream_t s);

// Error plumbing (thread-local message).
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define EVX_CUDA(call)                                   \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return ::evx::cuda_fail(_e, #call); \
  } while (0)

// Launch the search for one query (defined in evx_search.cu).
int launch_search(const GraphView &g, const MotifPlan &plan, const SearchArgs &args,
                  int grid, int block, cudaStream_t stream);
// Launch a persistent search over a table of queries (count mode); q0 is
// used when nq == 1.  Every query of the table has k edges.
int launch_table(const GraphView &g, const QueryDesc &q0, const LaunchArgs &la, int k, bool ps, int grid,
                 cudaStream_t stream);
int table_occupancy(int k, bool ps, int *blocks_per_sm);
// Whether a query with these kQ flags walks a pair run at some level (the
// kernels are compiled with and without that walk).
bool plan_pair_scan(const MotifPlan &plan, int qflags, bool enumerate);
// Max resident blocks per SM for a given motif size / mode / pair-run
// variant / constrained variant (cs) / block.
int search_occupancy(int k, bool enumerate, bool ps, bool cs, int block, int *blocks_per_sm);
// Whether search args carry constraints (the CS kernel variant runs them).
inline bool cons_any(const ConsArgs &c) { return c.node_ok || c.edge_ok || c.has_gap; }

// A constrained search (evx_constrained.cu).  prev_real[j] = the latest motif
// edge before j that is not an anti-edge (0 for j = 1).
struct ConsSearch {
  MotifPlan plan;
  int root_beg, root_end;
  int delta;
  unsigned anti_mask;                        // bit j: motif edge j is an anti-edge
  int prev_real[EVX_MAX_MOTIF_EDGES];
  int has_temporal;
  int temporal[EVX_MAX_MOTIF_EDGES];         // [j-1]: gap bound of motif edge j
  int has_filter;
  int exact_total;                           // enumerate: keep counting past the cap
  evx_program filter;                        // variables e_0 .. e_{k-1}
  const unsigned short *node_ok;             // [V] bit a: may be motif node a (null: all)
  const unsigned char *edge_ok;              // [E] edge predicate (null: all)
  const int *edge_feat;                      // [E] filter variables
  unsigned long long *count;                 // result / enumeration slot counter
  int *cursor;                               // next unclaimed root id
  int *stop;                                 // set when the enumeration cap is reached
  int *rows;                                 // [cap * k] original line ids
  long long cap;
};
int launch_constrained(const GraphView &g, const ConsSearch &s, bool enumerate, int grid, cudaStream_t st);
int cons_occupancy(int k, bool enumerate, int *blocks_per_sm);
int cons_block();
// Host check of a program's opcodes, stack use and variable indices.
int cons_check_program(const evx_program &p, int num_vars, const char *what);
// Node bit sets and edge flags from the predicates (no-ops for absent ones).
int cons_build_masks(const evx_constraints &c, int n, const int *node_feat, int V, const int *edge_feat,
                     int E, unsigned short *node_ok, unsigned char *edge_ok, int num_sms, cudaStream_t s);

// Build the pair index (defined in evx_pairs.cu); needs edges[] packed.
int build_pair_index(DeviceGraph &g, cudaStream_t s);

// Check the host-format arrays on the device before anything indexes with
// them (evx_graph.cu); returns EVX_ERR_INVALID with a message on bad input.
int validate_graph(int device, int64_t E, int64_t V, const int *eg_d, const int *out_v_d, const int *in_v_d,
                   const int *out_r_d, const int *in_r_d, cudaStream_t s);

// Build the packed device layout from the uploaded host-format arrays
// (defined in evx_graph.cu).
int pack_graph(DeviceGraph &g, const int *eg_d, const int *out_v_d, const int *in_v_d,
               const int *out_r_d, const int *in_r_d, const int *euid_d, cudaStream_t s);

}  // namespace evx

// The opaque graph handle of the C ABI.
struct evx_graph {
  evx::DeviceGraph g;
};
