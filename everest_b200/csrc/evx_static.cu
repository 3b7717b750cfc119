// Allocation-free counting: evx_count_static (include/everest_b200.h).
//
// Some callers cannot call cudaMalloc at query time: a process whose device
// memory is entirely reserved by another allocator (a framework's caching
// allocator, or a serving process that pre-reserves its memory budget), or
// code that must keep working when the device has no free memory left.  This
// entry point runs count queries on a graph that is already resident and
// writes the counts to caller memory, keeping its only scratch -- one count,
// one root cursor and one stop flag per query -- in the file-scope device
// array below.  It calls no cudaMalloc, cudaFree or other allocating routine.
//
// The array exists once per device that loads this library and lives until
// the process exits.  Its device address is looked up with
// cudaGetSymbolAddress the first time a device is used (that first call must
// come before any stream capture); the host-side name of the array is only a
// stand-in and is never passed to a kernel.  Every call shares the array and
// it keeps the previous call's contents, so each query's slot is reset on
// the stream before its search; calls whose work overlaps on the GPU (other
// streams or threads) race on it and must be serialised by the caller.
#include <climits>
#include <mutex>
#include <string>

#include "evx_internal.cuh"

namespace evx {
namespace {

// [0, MAX): per-query counts; [MAX, 2 MAX): per-query {root cursor, stop flag}
static __device__ __align__(256) unsigned long long g_static_scratch[2 * EVX_STATIC_MAX_QUERIES];

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
unsigned long long *g_static_ptr[kMaxDevices] = {};

__global__ void static_reset_kernel(int q, int beg) {
  g_static_scratch[q] = 0ull;
  int *cs = reinterpret_cast<int *>(&g_static_scratch[EVX_STATIC_MAX_QUERIES + q]);
  cs[0] = beg;
  cs[1] = 0;
}

int static_scratch(int device, unsigned long long **ptr) {
  if (device < 0 || device >= kMaxDevices) return fail(EVX_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_ptr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
    g_static_ptr[device] = static_cast<unsigned long long *>(p);
  }
  *ptr = g_static_ptr[device];
  return EVX_OK;
}

}  // namespace
}  // namespace evx

using namespace evx;

namespace evx {
namespace {

// Checks query q and fills its plan and launch arguments (scratch slots
// included); launches nothing.
int static_query(const DeviceGraph &g, const int *k, const int *mu, const int *mv, const int *delta,
                 int64_t beg, int64_t end, unsigned flags, unsigned long long *scratch, int sms, int q,
                 int off, MotifPlan *plan, SearchArgs *a, int *grid) {
  const int kq = k[q];
  if (kq < 2 || kq > EVX_MAX_MOTIF_EDGES) return fail(EVX_ERR_INVALID, "query motif edge count out of range");
  int rc = build_plan(kq, mu + off, mv + off, plan);
  if (rc) return rc;
  if (delta[q] < 0) return fail(EVX_ERR_INVALID, "delta must be non-negative");
  if ((int64_t)g.max_t + (int64_t)delta[q] > (int64_t)INT_MAX)
    return fail(EVX_ERR_OVERFLOW, "t + delta overflows int32");
  int64_t e = end < 0 ? g.num_edges - kq + 1 : end;
  if (e > g.num_edges) e = g.num_edges;
  int64_t b = beg < 0 ? 0 : beg;
  if (e < b) e = b;
  *a = SearchArgs{};
  a->root_beg = (int)b;
  a->root_end = (int)e;
  a->delta = delta[q];
  a->strict_ts = (flags & EVX_FLAG_STRICT_TS) ? 1 : 0;
  a->roots_per_fetch = 32;
  a->steal_interval = (flags & EVX_FLAG_NO_STEAL) ? 0 : 16;
  a->min_split = 2;
  a->enumerate = 0;
  a->tail_flags = tail_mode(*plan, flags, false);
  a->count = scratch + q;
  a->cursor = reinterpret_cast<int *>(scratch + EVX_STATIC_MAX_QUERIES + q);
  a->stop = a->cursor + 1;
  int bps = 0;
  rc = search_occupancy(kq, false, plan_pair_scan(*plan, a->tail_flags, false), false, 128, &bps);
  if (rc) return rc;
  if (bps < 1) bps = 1;
  *grid = bps * sms;
  if ((int64_t)a->root_end + (int64_t)*grid * 4 * 32 >= (int64_t)INT_MAX)
    return fail(EVX_ERR_OVERFLOW, "root cursor would overflow int32");
  return EVX_OK;
}

// Restores the caller's current device on every return path.
struct DeviceGuard {
  int saved = -1;
  DeviceGuard() {
    if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
  }
  ~DeviceGuard() {
    if (saved >= 0) cudaSetDevice(saved);
  }
};

}  // namespace
}  // namespace evx

// Every query is checked (motif, delta, overflow, occupancy) before the first
// launch, so a call that returns an error for a bad query has queued no work.
// Once launched, the call waits for its stream before it returns, on success
// and on a launch error alike.
extern "C" int evx_count_static(const evx_graph *gh, int nq, const int *k, const int *mu,
                                const int *mv, const int *delta, int64_t beg, int64_t end,
                                unsigned flags, void *stream, uint64_t *counts) {
  if (!gh || !k || !mu || !mv || !delta || !counts) return fail(EVX_ERR_INVALID, "null argument");
  if (nq < 1 || nq > EVX_STATIC_MAX_QUERIES)
    return fail(EVX_ERR_INVALID, "evx_count_static takes 1.." + std::to_string(EVX_STATIC_MAX_QUERIES) +
                                     " queries per call (its static scratch has that many slots); got " +
                                     std::to_string(nq));
  const DeviceGraph &g = gh->g;
  DeviceGuard guard;
  EVX_CUDA(cudaSetDevice(g.device));
  unsigned long long *scratch = nullptr;
  int rc = static_scratch(g.device, &scratch);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  int sms = 148;
  EVX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g.device));
  MotifPlan plan;
  SearchArgs a;
  int grid = 0;
  // pass 1: check every query; nothing is launched yet
  for (int q = 0, off = 0; q < nq; off += k[q], q++) {
    rc = static_query(g, k, mu, mv, delta, beg, end, flags, scratch, sms, q, off, &plan, &a, &grid);
    if (rc) return rc;
  }
  // pass 2: reset each query's slot and launch its search
  const GraphView view = g.view();
  for (int q = 0, off = 0; q < nq; off += k[q], q++) {
    rc = static_query(g, k, mu, mv, delta, beg, end, flags, scratch, sms, q, off, &plan, &a, &grid);
    if (!rc) {
      static_reset_kernel<<<1, 1, 0, s>>>(q, 0);  // the work queue counts root tiles from 0
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) rc = cuda_fail(e, "static_reset_kernel launch");
    }
    if (!rc && a.root_end > a.root_beg) {
      rc = launch_search(view, plan, a, grid, 128, s);
      if (!rc) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(e, "search launch");
      }
    }
    if (rc) {
      cudaStreamSynchronize(s);  // nothing of this call is left running on return
      return rc;
    }
  }
  EVX_CUDA(cudaMemcpyAsync(counts, scratch, sizeof(uint64_t) * (size_t)nq, cudaMemcpyDeviceToHost, s));
  EVX_CUDA(cudaStreamSynchronize(s));
  return EVX_OK;
}
