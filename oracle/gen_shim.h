// Host shim for the search kernel the reference generates per query
// (system/tmine/KernelGen.py with warpCentric, warpBalancing and
// tailExpansion off, so each CUDA thread is one root's sequential search).
// TEST INFRASTRUCTURE ONLY (oracle/ref_generated.py): the generated body is
// compiled for the host against these stand-ins.
#pragma once
#include <algorithm>
#include <cstdint>

namespace corelib {
struct TemporalEdge { int u, v, t; };  // include/data.h:27-29
struct MotifEdgeInfoV1 {              // include/data.h:33-40
  int baseNode, constraintNode;
  int mappedNodes;
  const int *arrR;
  const int *arrV;
  int io;
  bool newNode;
};
namespace data {}
}  // namespace corelib

struct gen_dim1 { unsigned x; };
static thread_local gen_dim1 gen_thread_idx = {0};
static thread_local gen_dim1 gen_block_idx = {0};
static const gen_dim1 gen_block_dim = {1};
#define threadIdx gen_thread_idx
#define blockIdx gen_block_idx
#define blockDim gen_block_dim
#define __device__
#define __global__
using std::min;

// one thread per block: the warp reduction adds nothing
template <class T> static inline T __shfl_down_sync(unsigned, T, int) { return T(0); }
static inline unsigned long long atomicAdd(unsigned long long *p, unsigned long long v) {
  return __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}
// The enumeration body stops the warp-centric root dispatcher with
// atomicExch(source, work) once the cap is reached; with one root per thread
// there is no dispatcher, so the fixtures keep every total under the cap.
static int gen_source_word = 0;
static int *source = &gen_source_word;
static inline int atomicExch(int *p, int v) { return __atomic_exchange_n(p, v, __ATOMIC_RELAXED); }
