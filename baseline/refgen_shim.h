// Stand-ins for the two reference headers that the generated per-query
// search file includes (include/helpers.cuh, include/data.h), so that the
// file KernelGen writes (system/tmine/KernelGen.py:112-151) and the legacy
// plugins (plugins/GPUWorker*.cu) compile for sm_100a without the
// reference's corelib host library, which needs Boost, range-v3 and a
// network fetch to build.
//
// The types keep the reference's field names and meaning:
//   TemporalEdge            include/data.h:27-29
//   MotifEdgeInfoV1         include/data.h:33-40
//   DeviceJobData, MineJob  include/data.h:304-336 (only the fields the
//                           generated worker reads)
//   GPUWorker               include/data.h:342-366, src/core/cpu/data.cc:529-569
// gpuErrchk throws instead of calling exit(), and so does the generated
// launch check's exit(-1), so that a failure reaches the caller as an
// error code instead of ending the process.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdio.h>
#include <thrust/device_ptr.h>
#include <thrust/functional.h>
#include <thrust/reduce.h>
#include <thrust/scan.h>

#include <climits>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

struct refgen_error : std::runtime_error {
  int code;
  refgen_error(int c, const std::string &what) : std::runtime_error(what), code(c) {}
};

inline void refgen_assert(cudaError_t code, const char *file, int line) {
  if (code != cudaSuccess)
    throw refgen_error((int)code, std::string(cudaGetErrorString(code)) + " at " + file + ":" +
                                      std::to_string(line));
}
#define gpuErrchk(ans) { refgen_assert((ans), __FILE__, __LINE__); }
// every header the generated file names is included above, before this
// macro exists (the build strips the generated file's own #include lines)
#define exit(code) throw refgen_error((code), "generated launch check failed")

// Tail-expansion offload buffer.  The reference sizes it for 2092 * 96
// contexts (system/templates/tailExpan/execMemInit.snp:5,11); one context is
// dumped per resident thread at most, and a B200 holds up to 148 SMs x 2048
// threads, so the build replaces the constant with this one.
#define REFGEN_OFFLOAD_CONTEXTS (4096 * 96)

// The expansion rounds prefix-sum the dumped widths in int
// (system/templates/tailExpan/Expanding.snp); a sum past INT_MAX would
// wrap and index outside the contexts.  The build inserts this check before
// that scan and refuses such a round instead.
#define REFGEN_CHECK_EXPAND(dev_ptr, cnt)                                                         \
  {                                                                                               \
    long long refgen_tot =                                                                        \
        thrust::reduce(dev_ptr, dev_ptr + (cnt), 0LL, thrust::plus<long long>());                 \
    if (refgen_tot > (long long)INT_MAX - (1LL << 24))                                            \
      throw refgen_error(-2, "tail-expansion width sum " + std::to_string(refgen_tot) +         \
                                 " overflows the reference's int prefix sum");                   \
  }

namespace corelib {
struct TemporalEdge {
  int u, v, t;
};
struct MotifEdgeInfoV1 {
  int baseNode, constraintNode;
  int mappedNodes;
  const int *arrR;
  const int *arrV;
  int io;
  bool newNode;
};
namespace data {
struct DeviceJobData {
  int device{0};
  size_t graphNumEdges{0}, graphNumVertices{0};
  const TemporalEdge *Eg_d{nullptr};
  const int *inEdgesV_d{nullptr}, *outEdgesV_d{nullptr}, *inEdgesR_d{nullptr}, *outEdgesR_d{nullptr};
  const int *edgefeatures_d{nullptr}, *nodefeatures_d{nullptr};
  const int *Euid_d{nullptr};
  size_t motifNumEdges{0}, motifNumVertices{0};
  const MotifEdgeInfoV1 *minfo_d{nullptr};
  const TemporalEdge *em_d{nullptr};  // motif edges {u, v, t} (HostMotifData::edges)
  const MotifEdgeInfoV1 *minfo() const { return minfo_d; }
  const TemporalEdge *Em_d() const { return em_d; }
};
struct MineJob {
  int device{-1};
  int beg{-1}, end{-1}, delta{-1};
  const DeviceJobData *data{nullptr};
};
}  // namespace data

struct GPUWorker {
  std::string type_;
  int gpu_;
  unsigned long long time_;
  int sizeBlock_;
  unsigned long long count_ = 0;
  data::MineJob *job_ = nullptr;
  GPUWorker(std::string type, int gpu = 0, int sizeBlock = 96)
      : type_(type), gpu_(gpu), time_(0), sizeBlock_(sizeBlock) {}
  virtual ~GPUWorker() {}
  virtual unsigned long long run() = 0;
  virtual void take(data::MineJob &job) { job_ = &job; }
  virtual void update_job() = 0;
  virtual std::vector<int> printEnum(int) { return {}; }
  unsigned long long count() const { return count_; }
  // src/core/cpu/data.cc:556-562: one thread per root of the job
  int numBlocks() const { return job_ ? (job_->end + sizeBlock_ - 1) / sizeBlock_ : -1; }
};
}  // namespace corelib
