// Host driver for the reference's legacy Baseline search body.  One OpenMP
// iteration plays one CUDA thread (one root edge id), exactly as the
// reference's grid of ceil(work/96) x 96 threads does.  TEST INFRASTRUCTURE
// ONLY (CPU baseline and cross-check).
#include "ref_shim.h"
#include "baseline_body.inc"

// Roots beg, beg + stride, beg + 2 stride, ... below end (stride 1: every
// root of the range; a larger stride samples the whole range evenly).
extern "C" int ref_baseline_count_strided(const int *eg_aos, int numeg,
                                          const int *in_v, const int *in_r,
                                          const int *out_v, const int *out_r,
                                          const int *em_aos, int numem, int numnm,
                                          int delta, int beg, int end, int stride, int nthreads,
                                          unsigned long long *count_out) {
  if (numnm > 5 || numem > 6) return -1;  // MapMg[5] / Estack[5] in the body
  if (stride < 1) return -2;
  unsigned long long gcount = 0;
  const TemporalEdge *Eg = reinterpret_cast<const TemporalEdge *>(eg_aos);
  const TemporalEdge *Em = reinterpret_cast<const TemporalEdge *>(em_aos);
  const long n = end > beg ? (end - beg + stride - 1) / stride : 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
  for (long i = 0; i < n; i++) {
    const long tid = beg + i * stride;
    evx_thread_idx.x = (unsigned)(tid % 96);
    evx_block_idx.x = (unsigned)(tid / 96);
    MotifMatching_dispatch(end, delta, Eg, numeg, in_v, in_r, out_v, out_r,
                           nullptr, Em, numem, numnm, &gcount);
  }
  *count_out = gcount;
  return 0;
}

extern "C" int ref_baseline_count(const int *eg_aos, int numeg,
                                  const int *in_v, const int *in_r,
                                  const int *out_v, const int *out_r,
                                  const int *em_aos, int numem, int numnm,
                                  int delta, int beg, int end, int nthreads,
                                  unsigned long long *count_out) {
  return ref_baseline_count_strided(eg_aos, numeg, in_v, in_r, out_v, out_r, em_aos, numem, numnm,
                                    delta, beg, end, 1, nthreads, count_out);
}
