// Runs the search the reference generates for one query -- the file that
// system/tmine/KernelGen.py:112-151 writes with warpCentric, warpBalancing
// and tailExpansion on, the configuration Everest ships -- or one of its
// legacy ablation plugins (plugins/GPUWorker*.cu), built for sm_100a,
// through its own GPUWorker (getWorker / take / run,
// system/templates/GPUWorker/*.snp).  A comparator for timing and a
// full-size parity check; the library of this repository never links it.
//
// REFGEN_BODY names the generated file after refgen.py stripped its
// #include lines and made the two changes refgen_shim.h describes (offload
// buffer size, int-overflow check before the expansion scan).
#include "refgen_shim.h"
#include REFGEN_BODY
#undef exit

#include <chrono>
#include <cstring>

namespace {

struct RefGraph {
  corelib::TemporalEdge *eg = nullptr;
  int *in_v = nullptr, *in_r = nullptr, *out_v = nullptr, *out_r = nullptr;
  int num_edges = 0, num_vertices = 0;
};

void put_error(char *err, int errlen, const std::string &s) {
  if (err && errlen > 0) {
    std::strncpy(err, s.c_str(), (size_t)errlen - 1);
    err[errlen - 1] = 0;
  }
}

}  // namespace

// Upload the reference's HostGraphData arrays (Eg AoS {u, v, t}, in/out edge
// lists, in/out offsets; src/core/gpu/data.cu:124-348) to device 0.  Every
// array gets kPad zeroed entries past its end: the legacy U0 and U1 plugins
// read Eg[tid] before they check tid < work, for tids up to one block (96)
// past the last root.
constexpr size_t kPad = 256;
extern "C" int refgen_graph_upload(const int *eg_aos, int num_edges, const int *in_v, const int *in_r,
                                   const int *out_v, const int *out_r, int num_vertices, void **out,
                                   char *err, int errlen) {
  RefGraph *g = new RefGraph();
  try {
    g->num_edges = num_edges;
    g->num_vertices = num_vertices;
    const size_t e = (size_t)(num_edges > 0 ? num_edges : 1) + kPad, nv = (size_t)num_vertices + 1 + kPad;
    gpuErrchk(cudaSetDevice(0));
    gpuErrchk(cudaMalloc(&g->eg, sizeof(corelib::TemporalEdge) * e));
    gpuErrchk(cudaMalloc(&g->in_v, sizeof(int) * e));
    gpuErrchk(cudaMalloc(&g->out_v, sizeof(int) * e));
    gpuErrchk(cudaMalloc(&g->in_r, sizeof(int) * nv));
    gpuErrchk(cudaMalloc(&g->out_r, sizeof(int) * nv));
    gpuErrchk(cudaMemset(g->eg, 0, sizeof(corelib::TemporalEdge) * e));
    gpuErrchk(cudaMemset(g->in_v, 0, sizeof(int) * e));
    gpuErrchk(cudaMemset(g->out_v, 0, sizeof(int) * e));
    gpuErrchk(cudaMemset(g->in_r, 0, sizeof(int) * nv));
    gpuErrchk(cudaMemset(g->out_r, 0, sizeof(int) * nv));
    gpuErrchk(cudaMemcpy(g->eg, eg_aos, sizeof(corelib::TemporalEdge) * (size_t)num_edges, cudaMemcpyHostToDevice));
    gpuErrchk(cudaMemcpy(g->in_v, in_v, sizeof(int) * (size_t)num_edges, cudaMemcpyHostToDevice));
    gpuErrchk(cudaMemcpy(g->out_v, out_v, sizeof(int) * (size_t)num_edges, cudaMemcpyHostToDevice));
    const size_t nr = (size_t)num_vertices + 1;  // the host offsets end here; the padding stays zero
    gpuErrchk(cudaMemcpy(g->in_r, in_r, sizeof(int) * nr, cudaMemcpyHostToDevice));
    gpuErrchk(cudaMemcpy(g->out_r, out_r, sizeof(int) * nr, cudaMemcpyHostToDevice));
  } catch (const refgen_error &x) {
    put_error(err, errlen, x.what());
    cudaFree(g->eg); cudaFree(g->in_v); cudaFree(g->out_v); cudaFree(g->in_r); cudaFree(g->out_r);
    delete g;
    return x.code ? x.code : -1;
  }
  *out = g;
  return 0;
}

extern "C" void refgen_graph_free(void *h) {
  RefGraph *g = static_cast<RefGraph *>(h);
  if (!g) return;
  cudaFree(g->eg); cudaFree(g->in_v); cudaFree(g->out_v); cudaFree(g->in_r); cudaFree(g->out_r);
  delete g;
}

// Count the query this library was generated for over roots [beg, end)
// (end < 0: every root, E - k + 1, as MineJob does, src/core/cpu/data.cc:452-457)
// reps times with one worker.  ms_out[r] = host milliseconds around run(),
// the reference's GPUWorker::timed_run convention (src/core/cpu/data.cc:534-542).
extern "C" int refgen_count(void *h, const int *mu, const int *mv, int k, int delta, int beg, int end,
                            int reps, unsigned long long *count_out, double *ms_out, char *err,
                            int errlen) {
  RefGraph *g = static_cast<RefGraph *>(h);
  if (!g || k < 2 || reps < 1) {
    put_error(err, errlen, "bad arguments");
    return -1;
  }
  // Motif info as HostMotifData builds it (src/core/cpu/data.cc:411-449) and
  // DeviceJobData binds it (src/core/gpu/data.cu:516-526); motif nodes are
  // numbered by first appearance, edge 0 is 0->1.
  std::vector<corelib::MotifEdgeInfoV1> mi;
  int node_max = 1;
  for (int i = 1; i < k; i++) {
    corelib::MotifEdgeInfoV1 m{};
    if (mu[i] > node_max) {
      m.baseNode = mv[i]; m.constraintNode = -mu[i]; m.io = 0; m.mappedNodes = node_max + 1;
      m.newNode = true; node_max++;
    } else if (mv[i] > node_max) {
      m.baseNode = mu[i]; m.constraintNode = -mv[i]; m.io = 1; m.mappedNodes = node_max + 1;
      m.newNode = true; node_max++;
    } else {
      m.baseNode = mv[i]; m.constraintNode = mu[i]; m.io = -1; m.mappedNodes = node_max + 1;
      m.newNode = false;
    }
    m.arrR = m.io == 1 ? g->out_r : g->in_r;
    m.arrV = m.io == 1 ? g->out_v : g->in_v;
    mi.push_back(m);
  }
  // motif edges {u, v, t} in time order (HostMotifData::edges; the legacy
  // U0 plugin reads them)
  std::vector<corelib::TemporalEdge> em;
  for (int i = 0; i < k; i++) em.push_back({mu[i], mv[i], i + 1});
  corelib::MotifEdgeInfoV1 *mi_d = nullptr;
  corelib::TemporalEdge *em_d = nullptr;
  corelib::GPUWorker *w = nullptr;
  int rc = 0;
  try {
    gpuErrchk(cudaSetDevice(0));
    gpuErrchk(cudaMalloc(&mi_d, sizeof(corelib::MotifEdgeInfoV1) * mi.size()));
    gpuErrchk(cudaMemcpy(mi_d, mi.data(), sizeof(corelib::MotifEdgeInfoV1) * mi.size(), cudaMemcpyHostToDevice));
    gpuErrchk(cudaMalloc(&em_d, sizeof(corelib::TemporalEdge) * em.size()));
    gpuErrchk(cudaMemcpy(em_d, em.data(), sizeof(corelib::TemporalEdge) * em.size(), cudaMemcpyHostToDevice));
    corelib::data::DeviceJobData dd;
    dd.device = 0;
    dd.graphNumEdges = (size_t)g->num_edges;
    dd.graphNumVertices = (size_t)g->num_vertices;
    dd.Eg_d = g->eg;
    dd.inEdgesV_d = g->in_v; dd.outEdgesV_d = g->out_v;
    dd.inEdgesR_d = g->in_r; dd.outEdgesR_d = g->out_r;
    dd.motifNumEdges = (size_t)k;
    dd.motifNumVertices = (size_t)node_max + 1;
    dd.minfo_d = mi_d;
    dd.em_d = em_d;
    corelib::data::MineJob job;
    job.device = 0;
    job.beg = beg < 0 ? 0 : beg;
    job.end = end < 0 ? g->num_edges - k + 1 : end;
    job.delta = delta;
    job.data = &dd;
    w = getWorker(0);
    // run() returns the worker's running total (its count buffer is zeroed
    // only by the constructor), so each repetition's count is a difference
    unsigned long long c = 0, total = 0;
    for (int r = 0; r < reps; r++) {
      w->take(job);
      auto t0 = std::chrono::steady_clock::now();
      unsigned long long now = w->run();
      auto t1 = std::chrono::steady_clock::now();
      if (ms_out) ms_out[r] = std::chrono::duration<double, std::milli>(t1 - t0).count();
      if (r > 0 && now - total != c) throw refgen_error(-3, "count differs between repetitions");
      c = now - total;
      total = now;
    }
    *count_out = c;
  } catch (const refgen_error &x) {
    put_error(err, errlen, x.what());
    rc = x.code ? x.code : -1;
  }
  if (rc == 0) delete w;  // its destructor throws on a CUDA error; leak it then
  cudaFree(mi_d);
  cudaFree(em_d);
  return rc;
}
