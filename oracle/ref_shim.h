// Macro shim that lets the reference's legacy Baseline CUDA search body
// (plugins/GPUWorkerBaseline.cu:21-206) compile as host C++.  TEST
// INFRASTRUCTURE ONLY: used by the CPU baseline leg of bench.py and by tests.
#pragma once
#include <cstdint>

struct TemporalEdge { int u, v, t; };   // include/data.h:27-29 layout

struct evx_dim1 { unsigned x; };
static thread_local evx_dim1 evx_thread_idx = {0};
static thread_local evx_dim1 evx_block_idx = {0};
static const evx_dim1 evx_block_dim = {96};  // reference block size (include/data.h:351)

#define threadIdx evx_thread_idx
#define blockIdx evx_block_idx
#define blockDim evx_block_dim
#define __device__
#define __global__

static inline unsigned long long atomicAdd(unsigned long long *p, unsigned long long v) {
  return __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}
