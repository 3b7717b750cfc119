// Runs one generated search body (GEN_BODY, extracted by ref_generated.py)
// over every root on the host, one OpenMP iteration per root (one CUDA
// thread of the reference's grid).  TEST INFRASTRUCTURE ONLY.
#include "gen_shim.h"
#include GEN_BODY

#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

// Motif info as HostMotifData builds it (src/core/cpu/data.cc:411-449) and
// DeviceJobData binds it (src/core/gpu/data.cu:516-526); motif nodes are
// numbered by first appearance.
extern "C" int gen_count(const int *eg, int numeg, const int *in_v, const int *in_r,
                         const int *out_v, const int *out_r, const int *node_feat,
                         const int *edge_feat, const int *mu, const int *mv, int k, int delta,
                         int work, int *rows, const int *euid, int nthreads,
                         unsigned long long *count_out) {
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
    m.arrR = m.io == 1 ? out_r : in_r;
    m.arrV = m.io == 1 ? out_v : in_v;
    mi.push_back(m);
  }
  unsigned long long gcount = 0;
  const corelib::TemporalEdge *Eg = reinterpret_cast<const corelib::TemporalEdge *>(eg);
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
  for (int tid = 0; tid < work; tid++) {
    gen_block_idx.x = (unsigned)tid;
#ifdef GEN_ENUM
    // rows of Euid (here the sorted edge ids) into rows[cap * k]
    MotifMatching_dispatch(work, delta, Eg, numeg, in_v, in_r, out_v, out_r, node_feat, edge_feat,
                           mi.data(), k, rows, euid, &gcount);
#else
    MotifMatching_dispatch(work, delta, Eg, numeg, in_v, in_r, out_v, out_r, node_feat, edge_feat,
                           mi.data(), k, &gcount);
#endif
  }
  *count_out = gcount;
  return 0;
}
