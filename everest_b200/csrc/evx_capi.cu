// C ABI: device graphs and search workers (include/everest_b200.h).
#include <climits>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "evx_internal.cuh"

namespace evx {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();  // clear a sticky launch error where possible
  return fail(e == cudaErrorMemoryAllocation ? EVX_ERR_NOMEM : EVX_ERR_CUDA, m);
}

int graph_t_range(DeviceGraph &g, int *scratch_d, cudaStream_t s);

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};
}  // namespace

cudaError_t dev_alloc(void **p, size_t bytes, int device, cudaStream_t s) {
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  cudaMemPool_t pool;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pools[device]) {
      cudaMemPoolProps props;
      std::memset(&props, 0, sizeof(props));
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = device;
      cudaError_t e = cudaMemPoolCreate(&g_pools[device], &props);
      if (e != cudaSuccess) return e;
      uint64_t keep = ~0ull;  // keep freed memory mapped for reuse
      e = cudaMemPoolSetAttribute(g_pools[device], cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) return e;
    }
    pool = g_pools[device];
  }
  return cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, s);
}

void dev_free(void *p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

// Decode a relabeled motif into the per-level plan (HostMotifData rules,
// src/core/cpu/data.cc:416-446).
int build_plan(int k, const int *mu, const int *mv, MotifPlan *plan) {
  if (k < 2 || k > EVX_MAX_MOTIF_EDGES)
    return fail(EVX_ERR_INVALID, "motif must have 2.." + std::to_string(EVX_MAX_MOTIF_EDGES) + " edges");
  if (mu[0] != 0 || mv[0] != 1)
    return fail(EVX_ERR_INVALID, "motif edge 0 must be (0, 1) after relabeling");
  std::memset(plan, 0, sizeof(*plan));
  plan->k = k;
  int nm = 2;
  for (int j = 1; j < k; j++) {
    const int a = mu[j], b = mv[j];
    if (a < 0 || b < 0 || a == b)
      return fail(EVX_ERR_INVALID, "motif edge " + std::to_string(j) + " is a self-loop or negative");
    const bool an = a >= nm, bn = b >= nm;
    if (an && bn)
      return fail(EVX_ERR_INVALID, "motif edge " + std::to_string(j) + " touches no mapped node");
    int kind;
    if (an) {
      if (a != nm) return fail(EVX_ERR_INVALID, "motif nodes are not numbered by first appearance");
      kind = 0;
    } else if (bn) {
      if (b != nm) return fail(EVX_ERR_INVALID, "motif nodes are not numbered by first appearance");
      kind = 1;
    } else {
      kind = 2;
    }
    plan->info[j - 1] = kind | (a << 4) | (b << 8) | (nm << 12);
    if (an || bn) nm++;
    if (nm > EVX_MAX_MOTIF_NODES)
      return fail(EVX_ERR_INVALID, "motif has too many nodes");
  }
  plan->n = nm;
  return EVX_OK;
}

// Range arithmetic on the pair index replaces the last level's scan (count
// mode) for a closing last edge: when it closes on two nodes mapped before
// the second-to-last edge (its pair is fixed per partial match:
// kQInlineLast), when it repeats the second-to-last edge's endpoints (its
// pair run is the one the matched edge sits in: kQSamePair; when it reverses
// them, the reverse pair's run located per edge: kQRevPair), and for a
// closing edge whose pair changes with every partial match: one lookup per
// partial match in the pair hash table (kQPairHash, the default) or, on
// request, in the per-node pair directory (kQPairDir).  kQNoPrune turns off
// the check of the closing edge's fixed endpoint before a task's scan, and
// kQNoBound the per-root window bound from the last edge's list.  A last
// edge that maps a new node is scanned, and past the first step of a window
// the rest is counted by range arithmetic (kQNewArith) unless asked not to.
int tail_mode(const MotifPlan &plan, unsigned flags, bool enumerate) {
  const int np = ((flags & EVX_FLAG_NO_CLOSING_PRUNE) ? kQNoPrune : 0) |
                 ((flags & EVX_FLAG_NO_ROOT_BOUND) ? kQNoBound : 0) |
                 ((flags & (EVX_FLAG_LIST_SCAN | EVX_FLAG_NO_PAIR_INDEX | EVX_FLAG_CLOSING_SCAN)) ? 0 : kQPairScan);
  const int k = plan.k;
  if (enumerate || (flags & EVX_FLAG_NO_PAIR_INDEX) || k < 2) return np;
  const int wl = plan.info[k - 2];
  if (plan_kind(wl) != 2) return np | ((flags & EVX_FLAG_NEW_SCAN) ? 0 : kQNewArith);
  const int nm_prev = (k >= 3) ? plan_nm(plan.info[k - 3]) : 2;
  if (plan_a(wl) < nm_prev && plan_b(wl) < nm_prev) return kQInlineLast | np;
  if (k >= 3) {
    const int wp = plan.info[k - 3];
    if (plan_a(wp) == plan_a(wl) && plan_b(wp) == plan_b(wl)) return kQSamePair | np;
    if (plan_a(wp) == plan_b(wl) && plan_b(wp) == plan_a(wl)) return kQRevPair | np;
    // the pair depends on the node the second-to-last edge maps
    if (flags & EVX_FLAG_PAIR_DIR) return kQPairDir | np;
    if (!(flags & EVX_FLAG_CLOSING_SCAN)) return kQPairHash | np;
  }
  return np;
}

}  // namespace evx

using namespace evx;

struct evx_worker {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 148;
  // small device state (u64 words): [0] count, [1] int cursor + int stop, [2] work meter
  unsigned long long *state_d = nullptr;
  unsigned long long *count_h = nullptr;  // pinned
  int *rows_d = nullptr;
  int64_t rows_cap = 0;  // allocated rows
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // bound job
  bool has_job = false;
  bool launched = false;
  GraphView view{};
  MotifPlan plan{};
  SearchArgs args{};
  int64_t enum_cap = 0;
  uint64_t last_count = 0;
  uint64_t limit = 0;  // work limit of later jobs (0 = none)
  // tuning
  int block = 256, blocks_per_sm = 0, roots_per_fetch = 32, steal_interval = 16, min_split = 2;
  int last_launches = 0;
  float last_ms = 0.f;
  // constrained job (evx_worker_take_constrained)
  bool cons_active = false;
  ConsSearch cons{};
  unsigned short *node_ok_d = nullptr;
  int64_t node_ok_cap = 0;
  unsigned char *edge_ok_d = nullptr;
  int64_t edge_ok_cap = 0;
};

extern "C" {

const char *evx_last_error(void) { return g_last_error.c_str(); }

int evx_device_mem_info(int device, int64_t *free_bytes, int64_t *total_bytes) {
  int ndev = 0;
  evx_device_count(&ndev);
  if (ndev == 0) return fail(EVX_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(EVX_ERR_INVALID, "bad device index");
  EVX_CUDA(cudaSetDevice(device));
  size_t fr = 0, tot = 0;
  EVX_CUDA(cudaMemGetInfo(&fr, &tot));
  if (free_bytes) *free_bytes = (int64_t)fr;
  if (total_bytes) *total_bytes = (int64_t)tot;
  return EVX_OK;
}

int evx_host_register(void *ptr, int64_t bytes) {
  if (!ptr || bytes <= 0) return fail(EVX_ERR_INVALID, "bad host range");
  EVX_CUDA(cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault));
  return EVX_OK;
}

int evx_host_unregister(void *ptr) {
  if (!ptr) return fail(EVX_ERR_INVALID, "null pointer");
  EVX_CUDA(cudaHostUnregister(ptr));
  return EVX_OK;
}

int evx_device_count(int *count) {
  if (!count) return fail(EVX_ERR_INVALID, "null count");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  *count = n;
  return EVX_OK;
}

static int alloc_graph(int device, int64_t E, int64_t V, evx_graph **out, cudaStream_t s) {
  if (!out) return fail(EVX_ERR_INVALID, "null output pointer");
  if (E < 0 || V < 0) return fail(EVX_ERR_INVALID, "negative sizes");
  // fewer than 2^30 edges: adjacency records keep positions in 30 bits
  // (kPosMask) beside two flag bits
  if (E >= INT_MAX / 2 || V >= INT_MAX - 1)
    return fail(EVX_ERR_OVERFLOW, "graph too large for int32 edge / vertex ids");
  int ndev = 0;
  evx_device_count(&ndev);
  if (ndev == 0) return fail(EVX_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(EVX_ERR_INVALID, "bad device index");
  EVX_CUDA(cudaSetDevice(device));
  evx_graph *h = new (std::nothrow) evx_graph();
  if (!h) return fail(EVX_ERR_NOMEM, "host allocation failed");
  DeviceGraph &g = h->g;
  g.device = device;
  g.num_edges = E;
  g.num_vertices = V;
  const size_t e1 = (size_t)(E > 0 ? E : 1);
  size_t bytes = 0;
  cudaError_t err = cudaSuccess;
  auto A = [&](void **p, size_t n) {
    if (err == cudaSuccess) { err = dev_alloc(p, n, device, s); bytes += n; }
  };
  A((void **)&g.edges, sizeof(int4) * e1);
  A((void **)&g.inpos, sizeof(int) * e1);
  A((void **)&g.euid, sizeof(int) * e1);
  A((void **)&g.out_rec, sizeof(int4) * e1);
  A((void **)&g.in_rec, sizeof(int4) * e1);
  A((void **)&g.node_rng, sizeof(int4) * (size_t)(V > 0 ? V : 1));
  g.bytes = (int64_t)bytes;
  if (err != cudaSuccess) {
    dev_free(g.edges, s); dev_free(g.inpos, s); dev_free(g.euid, s); dev_free(g.out_rec, s);
    dev_free(g.in_rec, s); dev_free(g.node_rng, s);
    delete h;
    return cuda_fail(err, "device graph allocation");
  }
  g.stream = s;
  *out = h;
  return EVX_OK;
}

static int finish_graph(evx_graph *h, cudaStream_t s) {
  int *scratch = nullptr;
  EVX_CUDA(dev_alloc((void **)&scratch, 2 * sizeof(int), h->g.device, s));
  int rc = graph_t_range(h->g, scratch, s);
  dev_free(scratch, s);
  if (!rc) rc = build_pair_index(h->g, s);
  if (!rc) {
    EVX_CUDA(cudaStreamSynchronize(s));
  }
  return rc;
}

int evx_graph_from_device(int device, int64_t num_edges, int64_t num_vertices, const int *eg_d,
                          const int *out_v_d, const int *in_v_d, const int *out_r_d,
                          const int *in_r_d, const int *euid_d, void *stream, evx_graph **out) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!out || (num_edges > 0 && (!eg_d || !out_v_d || !in_v_d)) || !out_r_d || !in_r_d)
    return fail(EVX_ERR_INVALID, "null graph array");
  int rc = alloc_graph(device, num_edges, num_vertices, out, s);
  if (rc) return rc;
  rc = validate_graph(device, num_edges, num_vertices, eg_d, out_v_d, in_v_d, out_r_d, in_r_d, s);
  if (!rc) rc = pack_graph((*out)->g, eg_d, out_v_d, in_v_d, out_r_d, in_r_d, euid_d, s);
  if (!rc) rc = finish_graph(*out, s);
  if (rc) { evx_graph_free(*out); *out = nullptr; }
  return rc;
}

int evx_graph_upload(int device, int64_t num_edges, int64_t num_vertices, const int *eg,
                     const int *out_v, const int *in_v, const int *out_r, const int *in_r,
                     const int *euid, void *stream, evx_graph **out) {
  if (!out || (num_edges > 0 && (!eg || !out_v || !in_v)) || !out_r || !in_r)
    return fail(EVX_ERR_INVALID, "null graph array");
  cudaStream_t s = (cudaStream_t)stream;
  if (num_edges < 0 || num_vertices < 0) return fail(EVX_ERR_INVALID, "negative sizes");
  int rc = alloc_graph(device, num_edges, num_vertices, out, s);
  if (rc) return rc;
  const size_t E = (size_t)(num_edges > 0 ? num_edges : 1), V1 = (size_t)num_vertices + 1;
  // staging in host-format layout (returned to the pool after packing)
  int *buf = nullptr;
  const size_t n_ints = 3 * E + E + E + V1 + V1 + E;
  cudaError_t err = dev_alloc((void **)&buf, n_ints * sizeof(int), device, s);
  if (err != cudaSuccess) {
    evx_graph_free(*out);
    *out = nullptr;
    return cuda_fail(err, "upload staging allocation");
  }
  int *eg_d = buf, *ov_d = eg_d + 3 * E, *iv_d = ov_d + E, *or_d = iv_d + E, *ir_d = or_d + V1,
      *eu_d = ir_d + V1;
  const size_t ne = (size_t)num_edges;
  rc = EVX_OK;
  auto C = [&](void *d, const void *h, size_t n) {
    if (rc == EVX_OK && n) {
      cudaError_t e = cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemcpyAsync(upload)");
    }
  };
  C(eg_d, eg, sizeof(int) * 3 * ne);
  C(ov_d, out_v, sizeof(int) * ne);
  C(iv_d, in_v, sizeof(int) * ne);
  C(or_d, out_r, sizeof(int) * V1);
  C(ir_d, in_r, sizeof(int) * V1);
  if (euid) C(eu_d, euid, sizeof(int) * ne);
  // the packing kernels index with these arrays: check them on the device first
  if (!rc) rc = validate_graph(device, num_edges, num_vertices, eg_d, ov_d, iv_d, or_d, ir_d, s);
  if (!rc) rc = pack_graph((*out)->g, eg_d, ov_d, iv_d, or_d, ir_d, euid ? eu_d : nullptr, s);
  dev_free(buf, s);
  if (!rc) rc = finish_graph(*out, s);
  cudaStreamSynchronize(s);
  if (rc) { evx_graph_free(*out); *out = nullptr; }
  return rc;
}

int evx_graph_free(evx_graph *h) {
  if (!h) return EVX_OK;
  DeviceGraph &g = h->g;
  cudaSetDevice(g.device);
  // like cudaFree, wait for work that may still read the graph, then return
  // its memory to the pool
  cudaDeviceSynchronize();
  cudaStream_t s = nullptr;  // the allocating stream may be gone; nothing is in flight now
  dev_free(g.edges, s); dev_free(g.inpos, s); dev_free(g.euid, s); dev_free(g.out_rec, s);
  dev_free(g.in_rec, s); dev_free(g.node_rng, s); dev_free(g.pair_tab, s); dev_free(g.pair_rec, s);
  dev_free(g.pair_loc, s); dev_free(g.pair_dir, s); dev_free(g.dir_off, s);
  dev_free(g.sig_out, s); dev_free(g.sig_in, s); dev_free(g.rev_loc, s);
  dev_free(g.cross_out, s); dev_free(g.cross_in, s);
  dev_free(g.node_feat, s); dev_free(g.edge_feat, s);
  cudaStreamSynchronize(s);
  delete h;
  return EVX_OK;
}

int evx_graph_info(const evx_graph *h, int64_t *num_edges, int64_t *num_vertices, int *device,
                   int64_t *device_bytes) {
  if (!h) return fail(EVX_ERR_INVALID, "null graph");
  if (num_edges) *num_edges = h->g.num_edges;
  if (num_vertices) *num_vertices = h->g.num_vertices;
  if (device) *device = h->g.device;
  if (device_bytes) *device_bytes = h->g.bytes;
  return EVX_OK;
}

int evx_worker_create(int device, void *stream, evx_worker **out) {
  if (!out) return fail(EVX_ERR_INVALID, "null output pointer");
  int ndev = 0;
  evx_device_count(&ndev);
  if (ndev == 0) return fail(EVX_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(EVX_ERR_INVALID, "bad device index");
  EVX_CUDA(cudaSetDevice(device));
  evx_worker *w = new (std::nothrow) evx_worker();
  if (!w) return fail(EVX_ERR_NOMEM, "host allocation failed");
  w->device = device;
  cudaDeviceGetAttribute(&w->num_sms, cudaDevAttrMultiProcessorCount, device);
  cudaError_t e = cudaSuccess;
  if (stream) {
    w->stream = (cudaStream_t)stream;
  } else {
    e = cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking);
    w->own_stream = true;
  }
  if (e == cudaSuccess) e = cudaMalloc(&w->state_d, 64);
  if (e == cudaSuccess) e = cudaMemset(w->state_d, 0, 64);
  if (e == cudaSuccess) e = cudaMallocHost(&w->count_h, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaEventCreate(&w->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&w->ev1);
  if (e != cudaSuccess) {
    evx_worker_destroy(w);
    return cuda_fail(e, "worker setup");
  }
  *out = w;
  return EVX_OK;
}

int evx_worker_destroy(evx_worker *w) {
  if (!w) return EVX_OK;
  cudaSetDevice(w->device);
  if (w->rows_d && w->stream) dev_free(w->rows_d, w->stream);
  if (w->node_ok_d && w->stream) dev_free(w->node_ok_d, w->stream);
  if (w->edge_ok_d && w->stream) dev_free(w->edge_ok_d, w->stream);
  if (w->stream) cudaStreamSynchronize(w->stream);
  cudaFree(w->state_d);
  if (w->count_h) cudaFreeHost(w->count_h);
  if (w->ev0) cudaEventDestroy(w->ev0);
  if (w->ev1) cudaEventDestroy(w->ev1);
  if (w->own_stream && w->stream) cudaStreamDestroy(w->stream);
  delete w;
  return EVX_OK;
}

int evx_worker_stream(evx_worker *w, void **stream) {
  if (!w || !stream) return fail(EVX_ERR_INVALID, "null argument");
  *stream = (void *)w->stream;
  return EVX_OK;
}

int evx_worker_set_tuning(evx_worker *w, int block, int blocks_per_sm, int roots_per_fetch,
                          int steal_interval, int min_split) {
  if (!w) return fail(EVX_ERR_INVALID, "null worker");
  if (block < 32 || block > 256 || block % 32)
    return fail(EVX_ERR_INVALID, "block must be a multiple of 32 in [32, 256]");
  if (blocks_per_sm < 0 || roots_per_fetch < 1 || roots_per_fetch > 4096 || steal_interval < 0 ||
      min_split < 2)
    return fail(EVX_ERR_INVALID, "bad tuning value");
  if (steal_interval & (steal_interval - 1))
    return fail(EVX_ERR_INVALID, "steal_interval must be 0 or a power of two");
  w->block = block;
  w->blocks_per_sm = blocks_per_sm;
  w->roots_per_fetch = roots_per_fetch;
  w->steal_interval = steal_interval;
  w->min_split = min_split;
  return EVX_OK;
}

// Grow the worker's enumeration buffer to enum_cap rows of k ids, admitted
// against free device memory.
static int ensure_rows(evx_worker *w, int64_t enum_cap, int k) {
  if (enum_cap <= 0) return EVX_OK;
  if (enum_cap > (int64_t)INT_MAX) return fail(EVX_ERR_INVALID, "enumeration cap too large");
  const int64_t need = enum_cap * (int64_t)k;
  if (need > w->rows_cap) {
    size_t fr = 0, tot = 0;
    EVX_CUDA(cudaMemGetInfo(&fr, &tot));
    const size_t bytes = (size_t)need * sizeof(int);
    const size_t reserve = (size_t)256 << 20;  // keep headroom for other work
    if (bytes + reserve > fr)
      return fail(EVX_ERR_NOMEM, "enumeration buffer of " + std::to_string(bytes) +
                                     " bytes not admitted (free " + std::to_string(fr) + ")");
    // stream-ordered pool memory: no device-wide synchronisation, so a
    // serving loop's other streams keep running while a buffer grows
    int64_t grow = need;
    if (2 * w->rows_cap > grow && (size_t)(2 * w->rows_cap) * sizeof(int) + reserve <= fr) grow = 2 * w->rows_cap;
    if (w->rows_d) { dev_free(w->rows_d, w->stream); w->rows_d = nullptr; w->rows_cap = 0; }
    EVX_CUDA(dev_alloc((void **)&w->rows_d, (size_t)grow * sizeof(int), w->device, w->stream));
    w->rows_cap = grow;
  }
  return EVX_OK;
}

int evx_worker_take(evx_worker *w, const evx_graph *gh, int k, const int *mu, const int *mv,
                    int delta, int64_t beg, int64_t end, int64_t enum_cap, unsigned flags) {
  if (!w || !gh || !mu || !mv) return fail(EVX_ERR_INVALID, "null argument");
  if (gh->g.device != w->device) return fail(EVX_ERR_INVALID, "graph and worker on different devices");
  MotifPlan plan;
  int rc = build_plan(k, mu, mv, &plan);
  if (rc) return rc;
  const DeviceGraph &g = gh->g;
  if (delta < 0) return fail(EVX_ERR_INVALID, "delta must be non-negative");
  if ((int64_t)g.max_t + (int64_t)delta > (int64_t)INT_MAX)
    return fail(EVX_ERR_OVERFLOW, "t + delta overflows int32 (max t " + std::to_string(g.max_t) +
                                      ", delta " + std::to_string(delta) + ")");
  const int64_t E = g.num_edges;
  if (end < 0) end = E - k + 1;
  if (end > E) end = E;
  if (beg < 0) beg = 0;
  if (end < beg) end = beg;
  EVX_CUDA(cudaSetDevice(w->device));
  rc = ensure_rows(w, enum_cap, k);
  if (rc) return rc;
  w->view = g.view();
  w->plan = plan;
  SearchArgs &a = w->args;
  std::memset(&a, 0, sizeof(a));
  a.root_beg = (int)beg;
  a.root_end = (int)end;
  a.delta = delta;
  a.strict_ts = (flags & EVX_FLAG_STRICT_TS) ? 1 : 0;
  a.roots_per_fetch = w->roots_per_fetch;
  a.steal_interval = (flags & EVX_FLAG_NO_STEAL) ? 0 : w->steal_interval;
  a.min_split = w->min_split;
  a.enumerate = enum_cap > 0 ? 1 : 0;
  a.tail_flags = tail_mode(plan, flags, enum_cap > 0);
  a.exact_total = (flags & EVX_FLAG_EXACT_TOTAL) ? 1 : 0;
  a.cap = enum_cap;
  a.rows = w->rows_d;
  a.count = w->state_d;
  a.cursor = reinterpret_cast<int *>(w->state_d + 1);
  a.stop = reinterpret_cast<int *>(w->state_d + 1) + 1;
  a.limit = (unsigned long long)w->limit;
  a.meter = w->state_d + 2;
  w->enum_cap = enum_cap;
  w->cons_active = false;
  w->has_job = true;
  w->launched = false;
  return EVX_OK;
}

int evx_graph_set_features(evx_graph *h, const int *node_features, const int *edge_features) {
  if (!h) return fail(EVX_ERR_INVALID, "null graph");
  DeviceGraph &g = h->g;
  EVX_CUDA(cudaSetDevice(g.device));
  auto put = [&](int **dst, const int *src, int64_t n) -> int {
    if (!src) return EVX_OK;
    if (!*dst) {
      EVX_CUDA(dev_alloc((void **)dst, sizeof(int) * (size_t)(n > 0 ? n : 1), g.device, nullptr));
      g.bytes += sizeof(int) * (n > 0 ? n : 1);
    }
    if (n > 0) EVX_CUDA(cudaMemcpyAsync(*dst, src, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, nullptr));
    return EVX_OK;
  };
  int rc = put(&g.node_feat, node_features, g.num_vertices);
  if (!rc) rc = put(&g.edge_feat, edge_features, g.num_edges);
  EVX_CUDA(cudaStreamSynchronize(nullptr));
  return rc;
}

int evx_worker_take_constrained(evx_worker *w, const evx_graph *gh, int k, const int *mu, const int *mv,
                                int delta, int64_t beg, int64_t end, int64_t enum_cap, unsigned flags,
                                const evx_constraints *c) {
  // nothing to check: the plain search (the same matches, and its tuned kernel)
  if (!c || (c->anti_mask == 0 && !c->has_temporal && c->node_mode == 0 && !c->has_edge && !c->has_filter))
    return evx_worker_take(w, gh, k, mu, mv, delta, beg, end, enum_cap, flags);
  if (!w || !gh || !mu || !mv) return fail(EVX_ERR_INVALID, "null argument");
  if (gh->g.device != w->device) return fail(EVX_ERR_INVALID, "graph and worker on different devices");
  if (flags & ~(EVX_FLAG_EXACT_TOTAL | EVX_FLAG_PER_LANE | EVX_FLAG_WARP_SYNC))
    return fail(EVX_ERR_INVALID,
                "constrained searches take no flag but EVX_FLAG_EXACT_TOTAL, EVX_FLAG_PER_LANE, EVX_FLAG_WARP_SYNC");
  MotifPlan plan;
  int rc = build_plan(k, mu, mv, &plan);
  if (rc) return rc;
  const DeviceGraph &g = gh->g;
  if (delta < 0) return fail(EVX_ERR_INVALID, "delta must be non-negative");
  if ((int64_t)g.max_t + (int64_t)delta > (int64_t)INT_MAX)
    return fail(EVX_ERR_OVERFLOW, "t + delta overflows int32");
  // anti-edges: never motif edge 0, 1 or k-1; both ends mapped by earlier real edges
  if (c->anti_mask >> k) return fail(EVX_ERR_INVALID, "anti-edge mask names edges past the motif");
  if (c->anti_mask & (1u | 2u | (1u << (k - 1))))
    return fail(EVX_ERR_INVALID, "motif edges 0, 1 and k-1 cannot be anti-edges");
  unsigned mapped = (1u << mu[0]) | (1u << mv[0]);
  ConsSearch cs;
  std::memset(&cs, 0, sizeof(cs));
  for (int j = 1; j < k; j++) {
    const bool anti = (c->anti_mask >> j) & 1;
    if (anti && !(((mapped >> mu[j]) & 1) && ((mapped >> mv[j]) & 1)))
      return fail(EVX_ERR_INVALID, "anti-edge " + std::to_string(j) + " touches a node no earlier real edge maps");
    if (!anti) mapped |= (1u << mu[j]) | (1u << mv[j]);
    int p = j - 1;
    while (p > 0 && ((c->anti_mask >> p) & 1)) p--;
    cs.prev_real[j] = p;
  }
  if (c->anti_mask && enum_cap > 0)
    return fail(EVX_ERR_INVALID, "enumeration with anti-edges is not supported (rows would name no edge)");
  if (c->has_temporal) {
    for (int j = 0; j < k - 1; j++) {
      const int64_t gap = c->temporal[j];
      if ((int64_t)g.max_t + gap > (int64_t)INT_MAX || (int64_t)g.min_t + gap < (int64_t)INT_MIN)
        return fail(EVX_ERR_OVERFLOW, "t + temporal gap overflows int32");
      cs.temporal[j] = (int)gap;
    }
  }
  if (c->node_mode < 0 || c->node_mode > 2) return fail(EVX_ERR_INVALID, "bad node_mode");
  if (c->node_mode) {
    if (!g.node_feat) return fail(EVX_ERR_STATE, "node predicates need node features on the graph");
    for (int a = 0; a < (c->node_mode == 1 ? 1 : plan.n); a++) {
      rc = cons_check_program(c->node[a], 1, "node predicate");
      if (rc) return rc;
    }
  }
  if (c->has_edge) {
    if (!g.edge_feat) return fail(EVX_ERR_STATE, "an edge predicate needs edge features on the graph");
    rc = cons_check_program(c->edge, 1, "edge predicate");
    if (rc) return rc;
  }
  if (c->has_filter) {
    if (!g.edge_feat) return fail(EVX_ERR_STATE, "a filter needs edge features on the graph");
    rc = cons_check_program(c->filter, k, "filter");
    if (rc) return rc;
    for (int i = 0; i < c->filter.len; i++)
      if ((c->filter.op[i] & 0x7f) == EVX_OP_VAR && ((c->anti_mask >> c->filter.arg[i]) & 1))
        return fail(EVX_ERR_INVALID, "the filter names an anti-edge");
  }
  const int64_t E = g.num_edges, V = g.num_vertices;
  if (end < 0) end = E - k + 1;
  if (end > E) end = E;
  if (beg < 0) beg = 0;
  if (end < beg) end = beg;
  EVX_CUDA(cudaSetDevice(w->device));
  rc = ensure_rows(w, enum_cap, k);
  if (rc) return rc;
  if (c->node_mode && V > w->node_ok_cap) {
    if (w->node_ok_d) { dev_free(w->node_ok_d, w->stream); w->node_ok_d = nullptr; w->node_ok_cap = 0; }
    EVX_CUDA(dev_alloc((void **)&w->node_ok_d, sizeof(unsigned short) * (size_t)V, w->device, w->stream));
    w->node_ok_cap = V;
  }
  if (c->has_edge && E > w->edge_ok_cap) {
    if (w->edge_ok_d) { dev_free(w->edge_ok_d, w->stream); w->edge_ok_d = nullptr; w->edge_ok_cap = 0; }
    EVX_CUDA(dev_alloc((void **)&w->edge_ok_d, (size_t)E, w->device, w->stream));
    w->edge_ok_cap = E;
  }
  rc = cons_build_masks(*c, plan.n, g.node_feat, (int)V, g.edge_feat, (int)E, w->node_ok_d, w->edge_ok_d,
                        w->num_sms, w->stream);
  if (rc) return rc;
  // Node and edge predicates and temporal gaps run on the warp-synchronous
  // search with the checks compiled in (the CS kernels), where range
  // arithmetic still counts closing last edges under node predicates alone
  // (on 7.8M edges, the 4-cycle with node predicates and gaps: 1.25 ms
  // against 2.17 ms per lane; with an edge predicate: 3.8 against 6.5 ms);
  // anti-edges and filters take the per-lane search, and EVX_FLAG_PER_LANE
  // sends any query there.
  const bool ws_ok = c->anti_mask == 0 && !c->has_filter && !(flags & EVX_FLAG_PER_LANE);
  if (ws_ok) {
    // Range arithmetic counts edges without looking at them, so it stays
    // only where no counted edge has a check: closing last edges under node
    // predicates alone.
    rc = evx_worker_take(w, gh, k, mu, mv, delta, beg, end, enum_cap, flags & EVX_FLAG_EXACT_TOTAL);
    if (rc) return rc;
    SearchArgs &a = w->args;
    a.limit = 0;  // no work limit on constrained jobs
    a.cons.node_ok = c->node_mode ? w->node_ok_d : nullptr;
    a.cons.edge_ok = c->has_edge ? w->edge_ok_d : nullptr;
    a.cons.has_gap = c->has_temporal ? 1 : 0;
    for (int j = 0; j < k - 1; j++) a.cons.gap[j] = cs.temporal[j];
    // (with gaps, a closing edge's window starts from the edge before it,
    // so the closing-endpoint check made with the level's own window is off)
    int tf = kQPairScan | (c->has_temporal ? kQNoPrune : 0);
    if (!c->has_edge && !c->has_temporal) tf |= tail_mode(plan, 0, enum_cap > 0) & ~kQNewArith;
    a.tail_flags = tf;
    return EVX_OK;
  }
  cs.plan = plan;
  cs.root_beg = (int)beg;
  cs.root_end = (int)end;
  cs.delta = delta;
  cs.anti_mask = c->anti_mask;
  cs.has_temporal = c->has_temporal ? 1 : 0;
  cs.has_filter = c->has_filter ? 1 : 0;
  cs.exact_total = (flags & EVX_FLAG_EXACT_TOTAL) ? 1 : 0;
  cs.filter = c->filter;
  cs.node_ok = c->node_mode ? w->node_ok_d : nullptr;
  cs.edge_ok = c->has_edge ? w->edge_ok_d : nullptr;
  cs.edge_feat = g.edge_feat;
  cs.count = w->state_d;
  cs.cursor = reinterpret_cast<int *>(w->state_d + 1);
  cs.stop = reinterpret_cast<int *>(w->state_d + 1) + 1;
  cs.rows = w->rows_d;
  cs.cap = enum_cap;
  w->view = g.view();
  w->plan = plan;
  std::memset(&w->args, 0, sizeof(w->args));  // no work limit on constrained jobs
  w->cons = cs;
  w->cons_active = true;
  w->enum_cap = enum_cap;
  w->has_job = true;
  w->launched = false;
  return EVX_OK;
}

namespace evx {
__global__ void reset_state_kernel(unsigned long long *count, int *cursor, int *stop, int beg) {
  *count = 0ull;
  *cursor = beg;  // the search's work queue: next unclaimed root tile
  *stop = 0;
  count[2] = 0ull;  // work meter
}
}  // namespace evx

// Launch of a job taken by evx_worker_take_constrained: state reset, then
// one constrained search over the job's roots.
static int launch_constrained_job(evx_worker *w) {
  ConsSearch &c = w->cons;
  int bps = w->blocks_per_sm;
  if (bps <= 0) {
    int rc = cons_occupancy(c.plan.k, w->enum_cap > 0, &bps);
    if (rc) return rc;
    if (bps <= 0) bps = 1;
  }
  const int grid = bps * w->num_sms;
  if ((int64_t)c.root_end + (int64_t)grid * cons_block() >= (int64_t)INT_MAX)
    return fail(EVX_ERR_OVERFLOW, "root cursor would overflow int32");
  reset_state_kernel<<<1, 1, 0, w->stream>>>(c.count, c.cursor, c.stop, c.root_beg);
  EVX_CUDA(cudaGetLastError());
  EVX_CUDA(cudaEventRecord(w->ev0, w->stream));
  int launches = 1;
  if (c.root_end > c.root_beg) {
    int rc = launch_constrained(w->view, c, w->enum_cap > 0, grid, w->stream);
    if (rc) return rc;
    launches++;
  }
  EVX_CUDA(cudaEventRecord(w->ev1, w->stream));
  EVX_CUDA(cudaMemcpyAsync(w->count_h, c.count, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                           w->stream));
  w->last_launches = launches;
  w->launched = true;
  return EVX_OK;
}

int evx_worker_launch(evx_worker *w) {
  if (!w) return fail(EVX_ERR_INVALID, "null worker");
  if (!w->has_job) return fail(EVX_ERR_STATE, "run before take");
  EVX_CUDA(cudaSetDevice(w->device));
  SearchArgs &a = w->args;
  int bps = w->blocks_per_sm;
  if (bps <= 0) {
    const int qf = (a.strict_ts ? kQStrict : 0) | a.tail_flags;
    const bool cs = cons_any(a.cons);
    int rc = search_occupancy(w->plan.k, a.enumerate != 0, cs || plan_pair_scan(w->plan, qf, a.enumerate != 0),
                              cs, w->block, &bps);
    if (rc) return rc;
    if (bps <= 0) bps = 1;
  }
  const int grid = bps * w->num_sms;
  const int64_t warps = (int64_t)grid * (w->block / 32);
  if ((int64_t)a.root_end + warps * (int64_t)a.roots_per_fetch >= (int64_t)INT_MAX)
    return fail(EVX_ERR_OVERFLOW, "root cursor would overflow int32");
  if (w->cons_active) return launch_constrained_job(w);
  reset_state_kernel<<<1, 1, 0, w->stream>>>(a.count, a.cursor, a.stop, 0);
  EVX_CUDA(cudaGetLastError());
  EVX_CUDA(cudaEventRecord(w->ev0, w->stream));
  int launches = 1;
  if (a.root_end > a.root_beg) {
    int rc = launch_search(w->view, w->plan, a, grid, w->block, w->stream);
    if (rc) return rc;
    EVX_CUDA(cudaGetLastError());
    launches++;
  }
  EVX_CUDA(cudaEventRecord(w->ev1, w->stream));
  EVX_CUDA(cudaMemcpyAsync(w->count_h, a.count, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                           w->stream));
  if (a.limit)
    EVX_CUDA(cudaMemcpyAsync(w->count_h + 1, a.meter, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             w->stream));
  w->last_launches = launches;
  w->launched = true;
  return EVX_OK;
}

int evx_worker_result(evx_worker *w, uint64_t *count) {
  if (!w || !count) return fail(EVX_ERR_INVALID, "null argument");
  if (!w->launched) return fail(EVX_ERR_STATE, "result before launch");
  EVX_CUDA(cudaSetDevice(w->device));
  EVX_CUDA(cudaStreamSynchronize(w->stream));
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, w->ev0, w->ev1) == cudaSuccess) w->last_ms = ms;
  w->last_count = *w->count_h;
  *count = w->last_count;
  w->launched = false;
  if (w->args.limit && w->count_h[1] > w->args.limit)
    return fail(EVX_ERR_LIMIT, "work limit " + std::to_string(w->args.limit) + " exceeded");
  return EVX_OK;
}

int evx_worker_set_limit(evx_worker *w, uint64_t max_work) {
  if (!w) return fail(EVX_ERR_INVALID, "null worker");
  w->limit = max_work;
  return EVX_OK;
}

int evx_worker_query(evx_worker *w, int *done) {
  if (!w || !done) return fail(EVX_ERR_INVALID, "null argument");
  if (!w->launched) return fail(EVX_ERR_STATE, "query before launch");
  cudaError_t e = cudaEventQuery(w->ev1);
  if (e == cudaErrorNotReady) { *done = 0; return EVX_OK; }
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventQuery");
  *done = 1;
  return EVX_OK;
}

int evx_worker_run(evx_worker *w, uint64_t *count) {
  int rc = evx_worker_launch(w);
  if (rc) return rc;
  return evx_worker_result(w, count);
}

int evx_worker_enum_rows(evx_worker *w, int64_t n, int *rows, int64_t *rows_written) {
  if (!w || (n > 0 && !rows)) return fail(EVX_ERR_INVALID, "null argument");
  if (!w->has_job || w->enum_cap <= 0) return fail(EVX_ERR_STATE, "no enumeration job");
  int64_t f = n;
  if ((int64_t)w->last_count < f) f = (int64_t)w->last_count;
  if (w->enum_cap < f) f = w->enum_cap;
  if (f < 0) f = 0;
  if (f > 0) {
    EVX_CUDA(cudaSetDevice(w->device));
    EVX_CUDA(cudaMemcpyAsync(rows, w->rows_d, sizeof(int) * (size_t)f * w->plan.k,
                             cudaMemcpyDeviceToHost, w->stream));
    EVX_CUDA(cudaStreamSynchronize(w->stream));
  }
  if (rows_written) *rows_written = f;
  return EVX_OK;
}

int evx_worker_last_stats(evx_worker *w, int *kernel_launches, float *device_ms) {
  if (!w) return fail(EVX_ERR_INVALID, "null worker");
  if (kernel_launches) *kernel_launches = w->last_launches;
  if (device_ms) *device_ms = w->last_ms;
  return EVX_OK;
}

}  // extern "C"
