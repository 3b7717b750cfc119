// Batched queries: many count queries against one resident graph in one
// persistent launch per motif size (include/everest_b200.h, evx_batch_*).
//
// The queries are ordered by motif size (stable); each size's queries form
// one device work queue: their root ranges are cut into tiles of tile_roots
// roots laid end to end, warps claim tiles with one atomicAdd and switch
// their per-warp query copy when a tile belongs to another query, so cheap
// and expensive queries share the GPU without per-query tails or per-query
// launches.  Each size runs the kernel instantiated for exactly that size
// (its levels are compile-time).  The launch sequence (query table upload,
// counter reset, the kernels, counts read-back) is captured once into a CUDA
// graph and replayed while the batch keeps the same shape.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "evx_internal.cuh"

using namespace evx;

struct evx_batch {
  int device = 0;
  int max_q = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  const evx_graph *graph = nullptr;
  std::vector<QueryDesc> queries;
  QueryDesc *table_d = nullptr;        // [max_q]
  QueryDesc *table_h = nullptr;        // pinned [max_q]
  unsigned long long *counts_d = nullptr;  // [max_q] counts, kCursors cursor words, [max_q] work meters
  unsigned long long *counts_h = nullptr;  // pinned [max_q] counts, [max_q] meters
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // tuning
  int tile_roots = 256, blocks_per_sm = 0, steal_interval = 16, min_split = 2, use_graph = 1;
  unsigned long long limit = 0;  // work limit per query (0 = none)
  // table order -> query index, and the motif-size groups of the table
  // (kGroupWords ints each)
  std::vector<int> order;
  std::vector<int> groups;
  // captured launch and the shape it was captured for
  cudaGraphExec_t exec = nullptr;
  std::vector<int> exec_groups;
  int exec_nq = -1, exec_tile_roots = -1;
  unsigned long long exec_limit = 0;
  const evx_graph *exec_graph = nullptr;
  bool launched = false;
  int last_launches = 0;
  float last_ms = 0.f;
};

namespace {

constexpr int kCursors = 8;  // one work-queue cursor word per motif size
// a motif-size group of the table: {k, first table position, queries, tiles,
// grid, pair-run walk (0/1)}
constexpr int kGroupWords = 6;

void drop_exec(evx_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->exec_nq = -1;
}

int enqueue(evx_batch *b, int nq) {
  unsigned long long *meter = b->counts_d + b->max_q + kCursors;
  EVX_CUDA(cudaMemcpyAsync(b->table_d, b->table_h, sizeof(QueryDesc) * (size_t)nq, cudaMemcpyHostToDevice,
                           b->stream));
  EVX_CUDA(cudaMemsetAsync(b->counts_d, 0, sizeof(unsigned long long) * (2 * (size_t)b->max_q + kCursors),
                           b->stream));
  for (size_t gi = 0; gi < b->groups.size(); gi += kGroupWords) {
    const int k = b->groups[gi], beg = b->groups[gi + 1], n = b->groups[gi + 2];
    const int tiles = b->groups[gi + 3], grid = b->groups[gi + 4];
    const bool ps = b->groups[gi + 5] != 0;
    if (tiles <= 0) continue;
    LaunchArgs la{};
    la.table = b->table_d + beg;
    la.nq = n;
    la.total_tiles = tiles;
    la.tile_roots = b->tile_roots;
    la.cursor = reinterpret_cast<int *>(b->counts_d + b->max_q + gi / kGroupWords);
    la.counts = b->counts_d + beg;
    la.limit = b->limit;
    la.meter = meter + beg;
    int rc = launch_table(b->graph->g.view(), b->table_h[beg], la, k, ps, grid, b->stream);
    if (rc) return rc;
    EVX_CUDA(cudaGetLastError());
  }
  EVX_CUDA(cudaMemcpyAsync(b->counts_h, b->counts_d, sizeof(unsigned long long) * (size_t)nq,
                           cudaMemcpyDeviceToHost, b->stream));
  if (b->limit)
    EVX_CUDA(cudaMemcpyAsync(b->counts_h + b->max_q, meter, sizeof(unsigned long long) * (size_t)nq,
                             cudaMemcpyDeviceToHost, b->stream));
  return EVX_OK;
}

}  // namespace

extern "C" {

int evx_batch_create(int device, int max_queries, void *stream, evx_batch **out) {
  if (!out) return fail(EVX_ERR_INVALID, "null output pointer");
  if (max_queries < 1 || max_queries > (1 << 20)) return fail(EVX_ERR_INVALID, "max_queries out of range");
  int ndev = 0;
  evx_device_count(&ndev);
  if (ndev == 0) return fail(EVX_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(EVX_ERR_INVALID, "bad device index");
  EVX_CUDA(cudaSetDevice(device));
  evx_batch *b = new (std::nothrow) evx_batch();
  if (!b) return fail(EVX_ERR_NOMEM, "host allocation failed");
  b->device = device;
  b->max_q = max_queries;
  cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
  cudaError_t e = cudaSuccess;
  if (stream) {
    b->stream = (cudaStream_t)stream;
  } else {
    e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    b->own_stream = true;
  }
  if (e == cudaSuccess) e = cudaMalloc(&b->table_d, sizeof(QueryDesc) * (size_t)max_queries);
  if (e == cudaSuccess) e = cudaMallocHost(&b->table_h, sizeof(QueryDesc) * (size_t)max_queries);
  if (e == cudaSuccess) e = cudaMalloc(&b->counts_d, sizeof(unsigned long long) * (2 * (size_t)max_queries + kCursors));
  if (e == cudaSuccess) e = cudaMallocHost(&b->counts_h, sizeof(unsigned long long) * 2 * (size_t)max_queries);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
  if (e != cudaSuccess) {
    evx_batch_destroy(b);
    return cuda_fail(e, "batch setup");
  }
  b->queries.reserve((size_t)max_queries);
  *out = b;
  return EVX_OK;
}

int evx_batch_destroy(evx_batch *b) {
  if (!b) return EVX_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_exec(b);
  cudaFree(b->table_d);
  cudaFree(b->counts_d);
  if (b->table_h) cudaFreeHost(b->table_h);
  if (b->counts_h) cudaFreeHost(b->counts_h);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return EVX_OK;
}

int evx_batch_clear(evx_batch *b) {
  if (!b) return fail(EVX_ERR_INVALID, "null batch");
  if (b->launched) return fail(EVX_ERR_STATE, "batch launched: read its result first");
  b->queries.clear();
  b->graph = nullptr;
  return EVX_OK;
}

int evx_batch_set_tuning(evx_batch *b, int tile_roots, int blocks_per_sm, int steal_interval, int min_split,
                         int use_graph, int reserved) {
  (void)reserved;
  if (!b) return fail(EVX_ERR_INVALID, "null batch");
  if (tile_roots < 32 || tile_roots % 32 || tile_roots > (1 << 20))
    return fail(EVX_ERR_INVALID, "tile_roots must be a multiple of 32 in [32, 2^20]");
  if (blocks_per_sm < 0 || steal_interval < 0 || (steal_interval & (steal_interval - 1)) || min_split < 2)
    return fail(EVX_ERR_INVALID, "bad tuning value");
  b->tile_roots = tile_roots;
  b->blocks_per_sm = blocks_per_sm;
  b->steal_interval = steal_interval;
  b->min_split = min_split;
  b->use_graph = use_graph ? 1 : 0;
  drop_exec(b);
  return EVX_OK;
}

int evx_batch_set_limit(evx_batch *b, uint64_t max_work) {
  if (!b) return fail(EVX_ERR_INVALID, "null batch");
  if (b->launched) return fail(EVX_ERR_STATE, "batch launched: read its result first");
  b->limit = max_work;
  return EVX_OK;
}

int evx_batch_add(evx_batch *b, const evx_graph *gh, int k, const int *mu, const int *mv, int delta, int64_t beg,
                  int64_t end, unsigned flags, int *index_out) {
  if (!b || !gh || !mu || !mv) return fail(EVX_ERR_INVALID, "null argument");
  if (b->launched) return fail(EVX_ERR_STATE, "batch launched: read its result first");
  if ((int)b->queries.size() >= b->max_q) return fail(EVX_ERR_INVALID, "batch is full");
  if (b->graph && b->graph != gh) return fail(EVX_ERR_INVALID, "all queries of a batch use one graph");
  if (gh->g.device != b->device) return fail(EVX_ERR_INVALID, "graph and batch on different devices");
  MotifPlan plan;
  int rc = build_plan(k, mu, mv, &plan);
  if (rc) return rc;
  const DeviceGraph &g = gh->g;
  if (delta < 0) return fail(EVX_ERR_INVALID, "delta must be non-negative");
  if ((int64_t)g.max_t + (int64_t)delta > (int64_t)INT_MAX)
    return fail(EVX_ERR_OVERFLOW, "t + delta overflows int32");
  const int64_t E = g.num_edges;
  if (end < 0) end = E - k + 1;
  if (end > E) end = E;
  if (beg < 0) beg = 0;
  if (end < beg) end = beg;
  QueryDesc q;
  std::memset(&q, 0, sizeof(q));
  q.plan = plan;
  q.root_beg = (int)beg;
  q.root_end = (int)end;
  q.delta = delta;
  q.flags = ((flags & EVX_FLAG_STRICT_TS) ? kQStrict : 0) | tail_mode(plan, flags, false);
  q.steal_interval = (flags & EVX_FLAG_NO_STEAL) ? 0 : b->steal_interval;
  q.min_split = b->min_split;
  b->graph = gh;
  b->queries.push_back(q);
  if (index_out) *index_out = (int)b->queries.size() - 1;
  return EVX_OK;
}

int evx_batch_launch(evx_batch *b) {
  if (!b) return fail(EVX_ERR_INVALID, "null batch");
  if (b->launched) return fail(EVX_ERR_STATE, "batch already launched");
  const int nq = (int)b->queries.size();
  if (nq == 0) return fail(EVX_ERR_STATE, "empty batch");
  EVX_CUDA(cudaSetDevice(b->device));
  // table order: by motif size, stable; one group (and one launch) per size
  b->order.resize(nq);
  for (int i = 0; i < nq; i++) b->order[i] = i;
  std::stable_sort(b->order.begin(), b->order.end(),
                   [b](int x, int y) { return b->queries[x].plan.k < b->queries[y].plan.k; });
  b->groups.clear();
  int launches = 0;
  for (int pos = 0; pos < nq;) {
    const int k = b->queries[b->order[pos]].plan.k;
    const int beg = pos;
    int tiles = 0;
    bool ps = false;
    for (; pos < nq && b->queries[b->order[pos]].plan.k == k; pos++) {
      QueryDesc q = b->queries[b->order[pos]];
      ps = ps || plan_pair_scan(q.plan, q.flags, false);
      q.tile_beg = tiles;
      const int n = q.root_end - q.root_beg;
      tiles += n > 0 ? (n + b->tile_roots - 1) / b->tile_roots : 0;
      b->table_h[pos] = q;
    }
    int bps = 0;
    int rc = table_occupancy(k, ps, &bps);  // also sets the kernel attributes before any capture
    if (rc) return rc;
    if (b->blocks_per_sm > 0) bps = b->blocks_per_sm;
    if (bps < 1) bps = 1;
    b->groups.insert(b->groups.end(), {k, beg, pos - beg, tiles, bps * b->num_sms, ps ? 1 : 0});
    launches += tiles > 0 ? 1 : 0;
  }
  if ((int)b->groups.size() / kGroupWords > kCursors)
    return fail(EVX_ERR_INVALID, "too many motif sizes in one batch");
  EVX_CUDA(cudaEventRecord(b->ev0, b->stream));
  if (b->use_graph) {
    if (!b->exec || b->exec_nq != nq || b->exec_groups != b->groups || b->exec_tile_roots != b->tile_roots ||
        b->exec_graph != b->graph || b->exec_limit != b->limit) {
      drop_exec(b);
      cudaGraph_t graph = nullptr;
      EVX_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      int rc = enqueue(b, nq);
      cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
      if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
      e = cudaGraphInstantiate(&b->exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) { b->exec = nullptr; return cuda_fail(e, "cudaGraphInstantiate"); }
      b->exec_nq = nq; b->exec_groups = b->groups;
      b->exec_tile_roots = b->tile_roots; b->exec_graph = b->graph; b->exec_limit = b->limit;
    }
    EVX_CUDA(cudaGraphLaunch(b->exec, b->stream));
  } else {
    int rc = enqueue(b, nq);
    if (rc) return rc;
  }
  EVX_CUDA(cudaEventRecord(b->ev1, b->stream));
  b->last_launches = launches;
  b->launched = true;
  return EVX_OK;
}

int evx_batch_result(evx_batch *b, uint64_t *counts, int n) {
  if (!b) return fail(EVX_ERR_INVALID, "null batch");
  if (!b->launched) return fail(EVX_ERR_STATE, "result before launch");
  EVX_CUDA(cudaSetDevice(b->device));
  EVX_CUDA(cudaStreamSynchronize(b->stream));
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess) b->last_ms = ms;
  b->launched = false;
  const int nq = (int)b->queries.size();
  if (counts) {
    for (int pos = 0; pos < nq; pos++) {
      const int i = b->order[pos];
      if (i < n)
        counts[i] = (b->limit && b->counts_h[b->max_q + pos] > b->limit) ? UINT64_MAX : b->counts_h[pos];
    }
  }
  return EVX_OK;
}

int evx_batch_query(evx_batch *b, int *done) {
  if (!b || !done) return fail(EVX_ERR_INVALID, "null argument");
  if (!b->launched) return fail(EVX_ERR_STATE, "query before launch");
  cudaError_t e = cudaEventQuery(b->ev1);
  if (e == cudaErrorNotReady) { *done = 0; return EVX_OK; }
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventQuery");
  *done = 1;
  return EVX_OK;
}

int evx_batch_run(evx_batch *b, uint64_t *counts, int n) {
  int rc = evx_batch_launch(b);
  if (rc) return rc;
  return evx_batch_result(b, counts, n);
}

int evx_batch_last_stats(evx_batch *b, int *kernel_launches, float *device_ms) {
  if (!b) return fail(EVX_ERR_INVALID, "null batch");
  if (kernel_launches) *kernel_launches = b->last_launches;
  if (device_ms) *device_ms = b->last_ms;
  return EVX_OK;
}

}  // extern "C"
