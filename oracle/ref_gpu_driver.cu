// Device build of the reference's legacy Baseline search kernel for sm_100a
// (plugins/GPUWorkerBaseline.cu lines 21-206, extracted where they lie by
// ref_baseline.mk into _ref/baseline_body.inc; nothing of it is copied into
// the repository).  One thread per root edge, grid ceil(work / 96) x 96 as
// the reference launches it (GPUWorkerBaseline.cu:207-240).  TEST
// INFRASTRUCTURE ONLY: a parity and speed comparator for tests; the product
// never links it.
#include <cuda_runtime.h>

struct TemporalEdge { int u, v, t; };  // include/data.h:27-29 layout

#include "baseline_body.inc"

// Count one motif over roots [0, work) with the reference's kernel; reps
// launches, *ms_out = the fastest (CUDA events).  Returns 0, -1 for a motif
// the kernel's fixed-size stacks cannot hold, or the CUDA error code.
extern "C" int ref_gpu_count(const int *eg_aos, int numeg, const int *in_v, const int *in_r,
                             const int *out_v, const int *out_r, int num_vertices, const int *em_aos,
                             int numem, int numnm, int delta, int work, int reps,
                             unsigned long long *count_out, float *ms_out) {
  if (numnm > 5 || numem > 6) return -1;  // MapMg[5] / Estack[5] in the kernel
  TemporalEdge *eg = nullptr, *em = nullptr;
  int *iv = nullptr, *ir = nullptr, *ov = nullptr, *orr = nullptr;
  unsigned long long *cnt = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaMalloc(&eg, sizeof(TemporalEdge) * (size_t)(numeg > 0 ? numeg : 1));
  if (e == cudaSuccess) e = cudaMalloc(&em, sizeof(TemporalEdge) * (size_t)numem);
  if (e == cudaSuccess) e = cudaMalloc(&iv, sizeof(int) * (size_t)(numeg > 0 ? numeg : 1));
  if (e == cudaSuccess) e = cudaMalloc(&ov, sizeof(int) * (size_t)(numeg > 0 ? numeg : 1));
  if (e == cudaSuccess) e = cudaMalloc(&ir, sizeof(int) * (size_t)(num_vertices + 1));
  if (e == cudaSuccess) e = cudaMalloc(&orr, sizeof(int) * (size_t)(num_vertices + 1));
  if (e == cudaSuccess) e = cudaMalloc(&cnt, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemcpy(eg, eg_aos, sizeof(TemporalEdge) * (size_t)numeg, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(em, em_aos, sizeof(TemporalEdge) * (size_t)numem, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(iv, in_v, sizeof(int) * (size_t)numeg, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(ov, out_v, sizeof(int) * (size_t)numeg, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(ir, in_r, sizeof(int) * (size_t)(num_vertices + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(orr, out_r, sizeof(int) * (size_t)(num_vertices + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  float best = 0.f;
  unsigned long long c = 0;
  for (int r = 0; r < reps && e == cudaSuccess; r++) {
    e = cudaMemset(cnt, 0, sizeof(unsigned long long));
    if (e != cudaSuccess) break;
    cudaEventRecord(e0);
    if (work > 0)
      MotifMatching_dispatch<<<(work + 95) / 96, 96>>>(work, delta, eg, numeg, iv, ir, ov, orr, nullptr, em,
                                                       numem, numnm, cnt);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess && (r == 0 || ms < best)) best = ms;
  }
  if (e == cudaSuccess) e = cudaMemcpy(&c, cnt, sizeof(c), cudaMemcpyDeviceToHost);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(eg); cudaFree(em); cudaFree(iv); cudaFree(ov); cudaFree(ir); cudaFree(orr); cudaFree(cnt);
  if (e != cudaSuccess) return (int)e;
  *count_out = c;
  *ms_out = best;
  return 0;
}
