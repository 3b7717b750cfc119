// corelib -- C++ host layer with the reference's class names and semantics
// (include/data.h of the reference), implemented over the C ABI in
// include/everest_b200.h.  The pybind11 module (corelib_module.cc) exposes
// it to Python as `corelib` / `corelib.data`, the names system/tmine/core.py
// imports; plugin_evx.cc exports the `getWorker` factory
// (system/templates/GPUWorker/interface.snp:1-7).
//
// Differences from the reference, by design:
//  * errors throw std::runtime_error (Python RuntimeError) or
//    std::invalid_argument (ValueError); nothing calls exit();
//  * one prebuilt plugin serves every motif: the motif is bound at take()
//    time from DeviceJobData, so no per-query code generation or nvcc;
//  * FeatureLoader accepts a missing random-feature file (only queries with
//    node / edge predicates or a filter need it);
//  * query constraints reach the worker as data (GPUWorker::setConstraints),
//    not as generated code;
//  * multi-GPU execution classes exist but refuse more than one device.
#pragma once

#include <cstdint>
#include <filesystem>
#include <memory>
#include <string>
#include <tuple>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../../../include/everest_b200.h"

namespace corelib {

struct TemporalEdge {
  int u, v, t;
};

// Per motif edge j >= 1 (include/data.h:33-40): base node, constraint node
// (negative = -new node), nodes mapped before the edge, list direction
// (1 out, 0 in, -1 resolved at run time), whether the edge maps a new node.
struct MotifEdgeInfoV1 {
  int baseNode, constraintNode;
  int mappedNodes;
  int io;
  bool newNode;
};

std::string check_evx(int rc, const char *what);

namespace data {

// Cache directory conventions (include/data.h:96-117): <dir>/<stem>/...
struct CacheDirectoryAccess {
  std::string name_;
  std::filesystem::path graphPath_, cacheDir_;
  explicit CacheDirectoryAccess(const std::filesystem::path &pathToGraph, bool create = true);
  std::filesystem::path cacheUPath() const { return cacheDir_ / "U.cache"; }
  std::filesystem::path cacheVPath() const { return cacheDir_ / "V.cache"; }
  std::filesystem::path cacheTPath() const { return cacheDir_ / "T.cache"; }
  std::filesystem::path cacheIDSPath() const { return cacheDir_ / "IDS.cache"; }
  std::filesystem::path cacheFEPath() const { return cacheDir_ / "EdgesFeatures"; }
  std::filesystem::path cacheFVVPath() const { return cacheDir_ / "VerticesFeaturesValue"; }
  std::filesystem::path cacheFVMPath() const { return cacheDir_ / "VerticesFeaturesMap"; }
  std::filesystem::path cacheGraphDirPath(size_t beg, size_t end) const;
  std::string name() const { return name_; }
};

// Loads the time-sorted edge list; caches U/V/T/IDS as raw int32 files in the
// reference's layout (src/core/cpu/data.cc:175-314).
class EdgeListLoader : public CacheDirectoryAccess {
 public:
  explicit EdgeListLoader(const std::filesystem::path &pathToGraph, bool useCache = true);
  size_t edgeListLength() const { return U_.size(); }
  const std::vector<int> &U() const { return U_; }
  const std::vector<int> &V() const { return V_; }
  const std::vector<int> &T() const { return T_; }
  const std::vector<int> &IDS() const { return IDS_; }

 private:
  std::vector<int> U_, V_, T_, IDS_;
};

// Random per-edge / per-vertex features (src/core/cpu/data.cc:316-343,
// src/core/gpu/data.cu:57-79): a raw int32 file whose first E values are the
// features of the time-sorted edges and whose first N values those of the N
// distinct vertex ids in ascending order.  Like the reference, the derived
// arrays are cached beside the edge-list cache (EdgesFeatures,
// VerticesFeaturesValue, VerticesFeaturesMap) and read from there when all
// three exist.  A missing or short file yields empty features (queries
// without node / edge predicates need none).
class FeatureLoader : public CacheDirectoryAccess {
 public:
  FeatureLoader(const EdgeListLoader *eloader, const std::filesystem::path &pathToRands);
  size_t edgeFeaturesLength() const { return edge_.size(); }
  size_t verticesFeaturesLength() const { return vertex_.size(); }
  const std::vector<int> &edgeFeatures() const { return edge_; }
  // feature of an input vertex id (0 when the file held no vertex features)
  int vertexFeature(int id) const;
  bool hasVertexFeatures() const { return !vertex_.empty(); }

 private:
  std::vector<int> edge_, vertex_, vertexIds_;
};

// The graph data for a subset [beg, end) of the edge list
// (include/data.h:174-186).
struct HostGraphData {
  std::string name;
  size_t beg{0}, end{0};
  size_t numEdges{0}, numVertices{0}, totalBytes{0};
  std::vector<int> Eg, inEdgesV, outEdgesV, inEdgesR, outEdgesR, Euid;
  std::vector<int> edgeFeatures, verticesFeatures;
};

struct SubPartition {
  int beg, end, n;
};
typedef std::vector<SubPartition> SubPartitionList;
typedef std::vector<HostGraphData> HostGraphDataList;

// Time-range partitioning with a delta halo (src/core/cpu/data.cc:345-369).
SubPartitionList divideList(const EdgeListLoader &eloader, int delta, int num);
void removeMinor(HostGraphDataList &complete);
void includeMinor(HostGraphDataList &major, HostGraphDataList &minor);

class GraphDataLoader : public CacheDirectoryAccess {
 public:
  GraphDataLoader(const EdgeListLoader *eloader, const FeatureLoader *floader);
  std::string name() const { return stem_; }
  // src/core/gpu/data.cu:124-348; cache=true reads/writes the per-range
  // directory <cache>/<name>-<beg>-<end>/{Eg,inEdgesV,...} as raw int32 files.
  HostGraphData createGraphData(size_t beg = 0, size_t end = 0, bool cache = true) const;
  HostGraphDataList createPartitionsData(const SubPartitionList &partitions) const;
  HostGraphDataList createPartitionsDataMajor(const SubPartitionList &partitions) const;
  HostGraphDataList createPartitionsDataMinor(const SubPartitionList &partitions) const;

 private:
  const EdgeListLoader *eloader_;
  const FeatureLoader *floader_;
  std::string stem_;
  bool isCached(size_t beg, size_t end) const;
  HostGraphData loadGraphData(size_t beg, size_t end) const;
};

// A graph resident on one device (include/data.h:239-247).
struct DeviceGraphData {
  int device{0};
  std::string name;
  size_t beg{0}, end{0};
  size_t numEdges{0}, numVertices{0}, totalBytes{0};
  std::shared_ptr<evx_graph> graph;  // owns the device memory
};

// Moves host graphs to devices (include/data.h:250-274).
struct GraphDataManager {
  virtual std::vector<DeviceGraphData> allocBatch(int allDevices,
                                                  const std::vector<const HostGraphData *> &hostGraphs) const = 0;
  virtual DeviceGraphData alloc(int device, const HostGraphData *hostGraph) const = 0;
  virtual void moveAsync(DeviceGraphData &deviceGraph, const HostGraphData &hostGraph, int device) const = 0;
  virtual void waitMove(int device) const = 0;
  virtual ~GraphDataManager() {}
};
std::unique_ptr<GraphDataManager> MakeGraphDataManager(int totalDevice);

// Motif on the host (include/data.h:279-288).
struct HostMotifData {
  std::string name;
  size_t numEdges{0}, numVertices{0};
  std::vector<TemporalEdge> edges;   // relabeled, sorted by t
  std::vector<MotifEdgeInfoV1> minfo;
  explicit HostMotifData(const std::filesystem::path &pathToMotif);
  HostMotifData() = default;
  static HostMotifData fromText(const std::string &text, const std::string &name = "motif");
};

// Job data on a device: the motif plus a borrowed device graph
// (include/data.h:299-318).
struct DeviceJobData {
  int device{0};
  size_t graphNumEdges{0}, graphNumVertices{0};
  size_t motifNumEdges{0}, motifNumVertices{0};
  std::shared_ptr<evx_graph> graph;
  std::vector<int> mu, mv;
  std::vector<MotifEdgeInfoV1> minfol_;
  DeviceJobData(const DeviceGraphData &deviceGraph, const HostMotifData &hostMotif);
  DeviceJobData() = default;
};

// A job: roots [beg, end) of the graph, delta (include/data.h:323-336).
struct MineJob {
  int device{-1};
  int beg{-1}, end{-1}, delta{-1};
  const DeviceJobData *data{nullptr};
  MineJob(const DeviceJobData *_data, int _delta, int _beg = 0, int _end = -1);
  MineJob() = default;
  std::tuple<int, int> getWork() const { return {beg, end}; }
  void setWork(int _beg, int _end) { beg = _beg; end = _end; }
};

}  // namespace data

// The worker ABI (include/data.h:342-366).  Field order and virtual order
// follow the reference so that a host built against either header sees the
// same fields.
struct GPUWorker {
  std::string type_;
  int gpu_;
  unsigned long long time_;
  int sizeBlock_;
  unsigned long long count_;

  data::MineJob *job_ = nullptr;

  GPUWorker(std::string type, int gpu = 0, int sizeBlock = 96);
  virtual ~GPUWorker();
  virtual unsigned long long run() = 0;
  virtual void take(data::MineJob &job);
  virtual void update_job() = 0;
  int numBlocks();

  unsigned long long timed_run();
  unsigned long long time() const { return time_; }
  unsigned long long count() const { return count_; }
  void clear_time() { time_ = 0; }

  virtual std::vector<int> printEnum(int n);
  virtual std::pair<int, int> pause();

  // Extensions beyond the reference interface (query options it compiles into
  // each generated plugin): enumeration cap (0 = count), EVX_FLAG_* bits,
  // and the autotuner's launch parameters.
  virtual void configure(long long enumCap, unsigned flags);
  virtual void setTuning(int block, int blocksPerSM, int rootsPerFetch, int stealInterval,
                         int minSplit);
  virtual double lastDeviceMs() const;
  virtual int lastKernelLaunches() const;
  // Query constraints (node / edge predicates, temporal gaps, anti-edges,
  // filters), which the reference compiles into each generated plugin;
  // nullptr clears them.  Applies from the next take().
  virtual void setConstraints(const evx_constraints *c);
};

// The B200 worker behind the plugin.
struct GPUWorkerEVX : public GPUWorker {
  explicit GPUWorkerEVX(int gpu, int sizeBlock = 256);
  ~GPUWorkerEVX() override;
  unsigned long long run() override;
  void take(data::MineJob &job) override;
  void update_job() override;
  std::vector<int> printEnum(int n) override;
  void configure(long long enumCap, unsigned flags) override;
  void setTuning(int block, int blocksPerSM, int rootsPerFetch, int stealInterval,
                 int minSplit) override;
  double lastDeviceMs() const override;
  int lastKernelLaunches() const override;
  void setConstraints(const evx_constraints *c) override;

 private:
  evx_worker *w_ = nullptr;
  bool hasCons_ = false;
  evx_constraints cons_{};
  long long enumCap_ = 0;
  unsigned flags_ = 0;
  int k_ = 0;
  bool bound_ = false;
};

// dlopen handle of a worker plugin (include/data.h:369-383).
struct LibHandle {
  typedef GPUWorker *(*FactoryType)(int);
  void *handle = nullptr;
  FactoryType getWorker = nullptr;
  explicit LibHandle(const std::string &libpath);
  LibHandle(LibHandle &&rhs) noexcept;
  LibHandle &operator=(LibHandle &&rhs) noexcept;
  LibHandle(const LibHandle &) = delete;
  ~LibHandle();
  std::string toString() const;
};

class GPUWorkerLibManager {
  std::unordered_map<std::string, LibHandle> table_;

 public:
  // name = the NAME in lib<NAME>.so (src/core/cpu/data.cc:611-625)
  void openLib(const std::string &libpath);
  void unloadLib(const std::string &lib);
  std::unique_ptr<GPUWorker> construct(const std::string &lib, int gpu);
  std::string toString() const;
};

// Single-GPU execution (include/data.h:407-427, src/core/cpu/data.cc:642-677).
class SingleGPUExecution {
 protected:
  int device_{0};
  GPUWorker *w_{nullptr};
  const data::HostGraphData *hostGraph_{nullptr};
  int n_{-1};
  const data::HostMotifData *hostMotif_{nullptr};
  const data::GraphDataManager *dataManager_{nullptr};
  data::DeviceJobData jobData_;
  data::MineJob job_;
  data::DeviceGraphData deviceGraph_;
  virtual void formJobData();

 public:
  SingleGPUExecution(const data::GraphDataManager *dataManager, int device = 0);
  virtual ~SingleGPUExecution() {}
  void setHostGraph(const data::HostGraphData *hostGraph, int n = -1);
  void setHostMotif(const data::HostMotifData *hostMotif);
  void setWorker(GPUWorker *w);
  virtual unsigned long long run(int delta);
};

class SingleGPUExecutionDiv : public SingleGPUExecution {
  int div_;

 public:
  SingleGPUExecutionDiv(const data::GraphDataManager *dataManager, int device = 0, int div = 64);
  unsigned long long run(int delta) override;
};

// The reference marks its pause variant reserved; this one runs to completion.
class SingleGPUExecutionPause : public SingleGPUExecution {
 public:
  using SingleGPUExecution::SingleGPUExecution;
};

void SingleGPURunBatch(const data::GraphDataManager *dataManager, data::HostGraphDataList &hostGraphs,
                       const data::HostMotifData *hostMotif, GPUWorker *w, int delta);

// Multi-GPU classes: one device only on this path.
class MultiGPUExecution {
 protected:
  int deviceNum_;
  std::vector<GPUWorker *> ws_;
  std::vector<const data::HostGraphData *> hostGraphs_;
  data::SubPartitionList parts_;
  const data::HostMotifData *hostMotif_{nullptr};
  const data::GraphDataManager *dataManager_{nullptr};

 public:
  MultiGPUExecution(const data::GraphDataManager *dataManager, int deviceNum);
  virtual ~MultiGPUExecution() {}
  void setHostGraphs(const data::HostGraphDataList &hostGraphs, const data::SubPartitionList &ps);
  void setHostMotif(const data::HostMotifData *hostMotif);
  void setWorkers(std::vector<GPUWorker *> &ws);
  virtual void run(int delta);
  int numDevice() const { return deviceNum_; }
};
struct MultiGPUExecutionNaive : MultiGPUExecution { using MultiGPUExecution::MultiGPUExecution; };
struct MultiGPUExecutionDyn : MultiGPUExecution { using MultiGPUExecution::MultiGPUExecution; };
struct MultiGPUExecutionDynPause : MultiGPUExecution { using MultiGPUExecution::MultiGPUExecution; };

unsigned long long allCount(std::vector<GPUWorker *> &ws);

}  // namespace corelib
