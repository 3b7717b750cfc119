// Host driver for the reference's legacy Baseline search body.  One OpenMP
// iteration plays one CUDA thread (one root edge id), exactly as the
// reference's grid of ceil(work/96) x 96 threads does.  TEST INFRASTRUCTURE
// ONLY (CPU baseline and cross-check).
#include "ref_shim.h"
#include "baseline_body.inc"

extern "C" int ref_baseline_count(const int *eg_aos, int numeg,
                                  const int *in_v, const int *in_r,
                                  const int *out_v, const int *out_r,
                                  const int *em_aos, int numem, int numnm,
                                  int delta, int beg, int end, int nthreads,
                                  unsigned long long *count_out) {
  if (numnm > 5 || numem > 6) return -1;  // MapMg[5] / Estack[5] in the body
  unsigned long long gcount = 0;
  const TemporalEdge *Eg = reinterpret_cast<const TemporalEdge *>(eg_aos);
  const TemporalEdge *Em = reinterpret_cast<const TemporalEdge *>(em_aos);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
  for (long tid = beg; tid < end; tid++) {
    evx_thread_idx.x = (unsigned)(tid % 96);
    evx_block_idx.x = (unsigned)(tid / 96);
    MotifMatching_dispatch(end, delta, Eg, numeg, in_v, in_r, out_v, out_r,
                           nullptr, Em, numem, numnm, &gcount);
  }
  *count_out = gcount;
  return 0;
}
